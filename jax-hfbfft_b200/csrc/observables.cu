// Nuclear observables from the densities (calculate_complete_observables,
// output.py:177-340, density part).  One block per isospin accumulates the
// grid sums in FP64 in a fixed order (first sum rho, x rho and the currents,
// then the second moments about that isospin's own centre of mass); one
// thread turns the sums into the observables (observables.cuh).
#include <math.h>
#include "hfb_ctx.cuh"
#include "observables.cuh"

namespace hfb {

namespace {

constexpr int kObsThreads = 1024;

// Deterministic block sum of ``v`` (every thread gets the result).
__device__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < kObsThreads / 32; ++w) t += red[w];
  return t;
}

__global__ void __launch_bounds__(kObsThreads) obs_moments_kernel(int n, const double* __restrict__ rho,
                                                                  const double* __restrict__ cur, double dx,
                                                                  double dy, double dz, double* sums) {
  __shared__ double red[kObsThreads / 32];
  const int iq = blockIdx.x;
  const size_t n3 = (size_t)n * n * n;
  const double* r = rho + (size_t)iq * n3;
  const double h = (n - 1) / 2.0;
  double s[7] = {0, 0, 0, 0, 0, 0, 0};
  for (size_t i = threadIdx.x; i < n3; i += kObsThreads) {
    const int x = (int)(i / ((size_t)n * n)), y = (int)((i / n) % n), z = (int)(i % n);
    const double v = r[i];
    s[0] += v;
    s[1] += (x - h) * dx * v;
    s[2] += (y - h) * dy * v;
    s[3] += (z - h) * dz * v;
    if (cur) {
      s[4] += cur[((size_t)iq * 3 + 0) * n3 + i];
      s[5] += cur[((size_t)iq * 3 + 1) * n3 + i];
      s[6] += cur[((size_t)iq * 3 + 2) * n3 + i];
    }
  }
  double t[kObsSums];
  for (int k = 0; k < 7; ++k) t[k] = block_sum(s[k], red);
  const double cx = t[1] / t[0], cy = t[2] / t[0], cz = t[3] / t[0];
  double m[6] = {0, 0, 0, 0, 0, 0};
  for (size_t i = threadIdx.x; i < n3; i += kObsThreads) {
    const int x = (int)(i / ((size_t)n * n)), y = (int)((i / n) % n), z = (int)(i % n);
    const double v = r[i];
    const double a = (x - h) * dx - cx, b = (y - h) * dy - cy, c = (z - h) * dz - cz;
    m[0] += a * a * v;
    m[1] += b * b * v;
    m[2] += c * c * v;
    m[3] += a * b * v;
    m[4] += a * c * v;
    m[5] += b * c * v;
  }
  for (int k = 0; k < 6; ++k) t[7 + k] = block_sum(m[k], red);
  if (threadIdx.x == 0)
    for (int k = 0; k < kObsSums; ++k) sums[iq * kObsSums + k] = t[k];
}

__global__ void obs_final_kernel(const double* sums, double wxyz, double nneut, double nprot, double* out) {
  obs_finalize(sums, wxyz, nneut, nprot, out);
}

}  // namespace

}  // namespace hfb

using namespace hfb;

extern "C" int hfb_observables(hfb_ctx_t ctx, const double* rho, const double* current, double nneut,
                               double nprot, double* out, void* stream) {
  if (!ctx || !rho || !out || !(nneut > 0.0) || !(nprot > 0.0)) return HFB_ERR_ARG;
  cudaStream_t st = as_stream(stream);
  double* sums = (double*)scratch(ctx, hfb_ctx_s::S_PART2, sizeof(double) * 2 * kObsSums);
  if (!sums) return HFB_ERR_ALLOC;
  obs_moments_kernel<<<2, kObsThreads, 0, st>>>(ctx->n, rho, current, ctx->d[0], ctx->d[1], ctx->d[2], sums);
  HFB_CHECK_LAUNCH();
  obs_final_kernel<<<1, 1, 0, st>>>(sums, ctx->wxyz, nneut, nprot, out);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}
