// Context creation: grid, dense derivative matrices, Coulomb Green's
// function, scratch arena and the device status latch.
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <atomic>
#include <vector>
#include <cudaTypedefs.h>
#include "hfb_ctx.cuh"

namespace hfb {

static std::atomic<unsigned long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
static thread_local int t_last_cuda_error = 0;
void note_cuda_error(int e) { t_last_cuda_error = e; }

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library)
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
    }
    return (PFN_cuTensorMapEncodeTiled_v12000)p;
  }();
  return fn;
}

bool encode_fp32_rows_map(CUtensorMap* m, const void* base, uint64_t row_floats, uint64_t rows, uint32_t box_rows) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc || !base || ((uintptr_t)base & 15) || rows == 0 || box_rows == 0 || box_rows > 256) return false;
  cuuint64_t dims[2] = {(cuuint64_t)row_floats, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)(row_floats * sizeof(float))};
  cuuint32_t box[2] = {32, box_rows};
  cuuint32_t es[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(base), dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int coulomb_init(hfb_ctx_s* c);  // skyrme.cu
int hpsi_tc_prepare(hfb_ctx_s* c);   // hpsi_tc.cu
int hpsi_bf3_prepare(hfb_ctx_s* c);  // hpsi_bf3.cu
int hpsi_dmma_prepare(hfb_ctx_s* c); // hpsi_dmma.cu

void* scratch(hfb_ctx_s* c, int s, size_t bytes) {
  if (s < 0 || s >= hfb_ctx_s::S_NSLOT) return nullptr;
  if (bytes == 0) bytes = 16;
  if (c->slot_bytes[s] >= bytes) return c->slot[s];
  if (c->slot[s]) {
    cudaDeviceSynchronize();
    cudaFree(c->slot[s]);
    c->slot[s] = nullptr;
    c->slot_bytes[s] = 0;
  }
  size_t want = bytes + bytes / 8;
  if (cudaMalloc(&c->slot[s], want) != cudaSuccess) {
    cudaGetLastError();
    c->slot[s] = nullptr;
    return nullptr;
  }
  c->slot_bytes[s] = want;
  return c->slot[s];
}

// Dense spectral derivative matrices, restating grids.py:36-61:
//   der1[a][b] = afac/(icn d) sum_{j=1}^{icn-1} j sin(j afac (b-a))
//                (the icn term vanishes: sin(pi (b-a)) = 0 in the reference's
//                 arithmetic up to rounding, kept for identical rounding)
//   der2[a][b] = -afac^2/(icn d^2) [sum_j j^2 cos(j afac (b-a)) + icn^2/2 cos(icn afac (b-a))]
static void dense_derivatives(int n, double d, std::vector<double>& d1, std::vector<double>& d2) {
  const int icn = (n + 1) / 2;
  const double afac = M_PI / icn;
  d1.assign((size_t)n * n, 0.0);
  d2.assign((size_t)n * n, 0.0);
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b) {
      const double g = (double)(b - a);
      double s1 = 0.0, s2 = 0.0;
      for (int j = 1; j < icn; ++j) {
        s1 += -j * sin(j * afac * g);
        s2 += (double)j * j * cos(j * afac * g);
      }
      d1[(size_t)a * n + b] = -afac * (s1 - 0.5 * icn * sin(icn * afac * g)) / (icn * d);
      d2[(size_t)a * n + b] = -(afac * afac) * (s2 + 0.5 * icn * icn * cos(icn * afac * g)) / (icn * d * d);
    }
}

}  // namespace hfb

using namespace hfb;

extern "C" int hfb_ctx_create(int nx, int ny, int nz, double dx, double dy, double dz, int periodic, int nstmax,
                              hfb_ctx_t* out) {
  if (!out) return HFB_ERR_ARG;
  *out = nullptr;
  if (nx != ny || ny != nz) return HFB_ERR_UNSUPPORTED_GRID;
  if (nx % 2 != 0) return HFB_ERR_ARG;        // grids.py:103-106
  if (dx * dy * dz <= 0.0) {                  // grids.py:108-113
    if (dx <= 0.0) return HFB_ERR_ARG;
    dy = dz = dx;
  }
  int ok = dispatch_n(nx, [](auto) { return HFB_OK; });
  if (ok != HFB_OK) return ok;
  hfb_ctx_s* c = (hfb_ctx_s*)calloc(1, sizeof(hfb_ctx_s));
  if (!c) return HFB_ERR_ALLOC;
  c->n = nx;
  c->d[0] = dx; c->d[1] = dy; c->d[2] = dz;
  c->wxyz = dx * dy * dz;
  c->periodic = periodic ? 1 : 0;
  c->nstmax = nstmax;
  if (cudaGetDevice(&c->device) != cudaSuccess) {
    cudaGetLastError();
    free(c);
    return HFB_ERR_CUDA;
  }
  c->n2 = periodic ? nx : 2 * nx;
  {
    const char* e = getenv("HFB_NO_TCGEN05");
    c->use_tcgen05 = (e && e[0] == '1') ? 0 : 1;
    const char* j = getenv("HFB_LAMBDA_JACOBI");
    c->lambda_refine = (j && j[0] == '1') ? 0 : 1;
    // single-precision hpsi kernel: bf16x3 (default), tf32x3 or fft (HFB_HPSI_KERNEL)
    const char* h = getenv("HFB_HPSI_KERNEL");
    c->hpsi_kind = (h && strcmp(h, "tf32x3") == 0) ? 1 : (h && strcmp(h, "fft") == 0) ? 2 : 0;
    // FP64 Gram and rotation on the FP64 tensor cores unless HFB_F64_MMA=0
    const char* gk = getenv("HFB_F64_MMA");
    c->f64_mma = (gk && gk[0] == '0') ? 0 : 1;
    // single-precision rotation fed by TMA unless HFB_TMA_FEED=0
    // FP64 hpsi on the FP64 tensor cores unless HFB_F64_HPSI=fft
    const char* fh = getenv("HFB_F64_HPSI");
    c->f64_hpsi = (fh && strcmp(fh, "fft") == 0) ? 0 : 1;
    const char* gt = getenv("HFB_TMA_FEED");
    c->tma_feed = (gt && gt[0] == '0') ? 0 : 1;
    // H and G Gram matrices computed while the lambda eigensolve runs unless HFB_GRAM_SPLIT=0
    const char* gs = getenv("HFB_GRAM_SPLIT");
    c->gram_split = (gs && gs[0] == '0') ? 0 : 1;
    c->wait_limit = kDefaultWaitLimit;
    c->timeout_probe = 0;
  }
  const size_t nn = (size_t)nx * nx;
  for (int a = 0; a < 3; ++a) {
    std::vector<double> d1, d2;
    dense_derivatives(nx, c->d[a], d1, d2);
    if (cudaMalloc(&c->der1[a], nn * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&c->der2[a], nn * sizeof(double)) != cudaSuccess) {
      hfb_ctx_destroy(c);
      return HFB_ERR_ALLOC;
    }
    cudaMemcpy(c->der1[a], d1.data(), nn * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(c->der2[a], d2.data(), nn * sizeof(double), cudaMemcpyHostToDevice);
  }
  if (cudaMalloc(&c->dev_status, sizeof(int)) != cudaSuccess) {
    hfb_ctx_destroy(c);
    return HFB_ERR_ALLOC;
  }
  cudaMemset(c->dev_status, 0, sizeof(int));
  if (cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    c->side = nullptr;
  }
  // the second side stream is optional: without it Newton-Schulz stays on
  // the calling stream
  c->side2 = nullptr;
  c->ev_fork2 = c->ev_join2 = nullptr;
  if (cudaStreamCreateWithFlags(&c->side2, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_fork2, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_join2, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    if (c->ev_fork2) cudaEventDestroy(c->ev_fork2);
    if (c->side2) cudaStreamDestroy(c->side2);
    c->side2 = nullptr;
    c->ev_fork2 = c->ev_join2 = nullptr;
  }
  const size_t n2c = (size_t)c->n2 * c->n2 * c->n2;
  if (cudaMalloc(&c->coul_q, n2c * sizeof(double2)) != cudaSuccess) {
    hfb_ctx_destroy(c);
    return HFB_ERR_ALLOC;
  }
  int r = coulomb_init(c);
  if (r == HFB_OK) r = hpsi_tc_prepare(c);
  if (r == HFB_OK) r = hpsi_bf3_prepare(c);
  if (r == HFB_OK) r = hpsi_dmma_prepare(c);
  if (r == HFB_OK && cudaDeviceSynchronize() != cudaSuccess) r = HFB_ERR_CUDA;
  if (r != HFB_OK) {
    hfb_ctx_destroy(c);
    return r;
  }
  *out = c;
  return HFB_OK;
}

extern "C" int hfb_ctx_destroy(hfb_ctx_t c) {
  if (!c) return HFB_OK;
  cudaDeviceSynchronize();
  for (int a = 0; a < 3; ++a) {
    if (c->der1[a]) cudaFree(c->der1[a]);
    if (c->der2[a]) cudaFree(c->der2[a]);
  }
  if (c->coul_q) cudaFree(c->coul_q);
  if (c->hpsi_b) cudaFree(c->hpsi_b);
  if (c->hpsi_bf3_b) cudaFree(c->hpsi_bf3_b);
  if (c->hpsi_d64) cudaFree(c->hpsi_d64);
  if (c->dev_status) cudaFree(c->dev_status);
  if (c->side) {
    cudaStreamDestroy(c->side);
    cudaEventDestroy(c->ev_fork);
    cudaEventDestroy(c->ev_join);
  }
  if (c->side2) {
    cudaStreamDestroy(c->side2);
    cudaEventDestroy(c->ev_fork2);
    cudaEventDestroy(c->ev_join2);
  }
  for (int s = 0; s < hfb_ctx_s::S_NSLOT; ++s)
    if (c->slot[s]) cudaFree(c->slot[s]);
  free(c);
  return HFB_OK;
}

extern "C" unsigned long long hfb_launch_count(void) { return hfb::g_launches.load(); }

extern "C" const char* hfb_last_cuda_error(int* code) {
  const int e = hfb::t_last_cuda_error;
  if (code) *code = e;
  return e ? cudaGetErrorString((cudaError_t)e) : "no CUDA error";
}

extern "C" const char* hfb_status_string(int s) {
  switch (s) {
    case HFB_OK: return "ok";
    case HFB_ERR_ARG: return "invalid argument";
    case HFB_ERR_UNSUPPORTED_GRID: return "unsupported grid (cubic n in {8,16,24,32,40,48})";
    case HFB_ERR_CUDA: return "CUDA error";
    case HFB_ERR_NOT_BRACKETED: return "BCS particle number not bracketed on [-100, 100]";
    case HFB_ERR_NO_CONVERGENCE: return "iteration limit reached (Jacobi / Newton-Schulz / Brent)";
    case HFB_ERR_NONFINITE: return "non-finite value";
    case HFB_ERR_ALLOC: return "device allocation failed";
    case HFB_ERR_TIMEOUT: return "a bounded device wait ran out (tensor-core pipeline)";
    default: return "unknown status";
  }
}

extern "C" int hfb_set_wait_limit(hfb_ctx_t c, long long cycles) {
  if (!c || cycles <= 0) return HFB_ERR_ARG;
  c->wait_limit = cycles;
  return HFB_OK;
}

extern "C" int hfb_set_hpsi_kernel(hfb_ctx_t c, int kind) {
  if (!c || kind < 0 || kind > 2) return HFB_ERR_ARG;
  c->hpsi_kind = kind;
  return HFB_OK;
}

extern "C" int hfb_arm_timeout_probe(hfb_ctx_t c) {
  if (!c) return HFB_ERR_ARG;
  c->timeout_probe = 1;
  return HFB_OK;
}

extern "C" int hfb_device_status(hfb_ctx_t c, void* stream, int* status_out) {
  if (!c || !status_out) return HFB_ERR_ARG;
  int h = 0;
  cudaStream_t st = as_stream(stream);
  if (cudaMemcpyAsync(&h, c->dev_status, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return HFB_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return HFB_ERR_CUDA;
  if (h) cudaMemsetAsync(c->dev_status, 0, sizeof(int), st);
  *status_out = h;
  return HFB_OK;
}
