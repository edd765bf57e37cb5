// Library context: grid, device constants and the scratch arena.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include "../../include/hfb.h"
#include "hfb_common.cuh"

struct hfb_ctx_s {
  int n;                 // cubic grid size
  double d[3];           // spacings dx, dy, dz
  double wxyz;
  int periodic;
  int nstmax;
  int device;            // CUDA device current when the context was created
  int n2;                // Coulomb grid size (2n, or n when periodic)
  double* der1[3];       // dense spectral derivative matrices (grids.py:36-61)
  double* der2[3];
  double2* coul_q;       // Green's function in k space, n2^3 (coulomb.py:23-52)
  int* dev_status;       // latched device-side error code
  cudaStream_t side;     // secondary stream for independent work inside a call
  int use_tcgen05;       // single-precision contractions on the tensor cores (default 1;
                         // HFB_NO_TCGEN05=1 in the environment at creation selects CUDA cores)
  int lambda_refine;     // FP64 diagstep diagonalises lambda by eigen refinement (default 1;
                         // HFB_LAMBDA_JACOBI=1 at creation selects the Jacobi solver)
  cudaEvent_t ev_fork, ev_join;
  cudaStream_t side2;    // a second one (Newton-Schulz beside the eigensolve and the H, G Gram)
  cudaEvent_t ev_fork2, ev_join2;
  unsigned char* hpsi_b; // single-precision hpsi (tf32 kernel): derivative matrices in the tensor-core tile layout
  unsigned char* hpsi_bf3_b; // single-precision hpsi (bf16 three-term kernel): the same, bf16 h/m/l tiles
  int hpsi_kind;         // single-precision hpsi kernel: 0 bf16 three-term (default), 1 tf32 three-term, 2 FFT
                         // on CUDA cores (HFB_HPSI_KERNEL=bf16x3 / tf32x3 / fft at creation, hfb_set_hpsi_kernel)
  int f64_mma;           // FP64 Gram and rotation on the FP64 tensor cores (default; HFB_F64_MMA=0: CUDA cores)
  int f64_hpsi;          // FP64 hpsi: 1 FP64 tensor cores (default), 0 FFT kernels (HFB_F64_HPSI=fft at creation)
  double* hpsi_d64;      // FP64 hpsi on the tensor cores: D of each axis, [3][n][n] doubles
  int tma_feed;          // single-precision rotation: K blocks by TMA, A in TMEM (default; HFB_TMA_FEED=0 at
                         // creation: producers that load through registers)
  long long wait_limit;  // clock cycles any one bounded device wait may take (hfb_set_wait_limit)
  int timeout_probe;     // the next tensor-core hpsi launch runs its timeout path (hfb_arm_timeout_probe)
  int gram_split;        // diagstep: H, G Gram matrices after the lambda eigensolve's fork (HFB_GRAM_SPLIT)
  // scratch arena: fixed slots, grown on demand (never shrunk)
  enum { S_PART = 0, S_PART2, S_POIS, S_DENS, S_DERIV, S_GRAM, S_MAT, S_SMALL, S_RED, S_EIG, S_ROT, S_HPT, S_LAST, S_NAT, S_RESP, S_RESP2, S_VJP, S_ROT2, S_NSLOT };
  void* slot[S_NSLOT];
  size_t slot_bytes[S_NSLOT];
};

namespace hfb {

// Default bound of any one device-side wait of the tensor-core pipelines
// (about one second at the B200's clocks); hfb_set_wait_limit changes it.
constexpr long long kDefaultWaitLimit = 2000000000LL;

// Scratch buffer ``s`` of at least ``bytes``; nullptr on allocation failure.
void* scratch(hfb_ctx_s* c, int s, size_t bytes);

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Counts every kernel launch of the library (reported by hfb_launch_count).
// Allow a kernel all the dynamic shared memory the device opts in to (the
// opt-in maximum less the kernel's static shared memory).  Every call sets
// the same value for a kernel, so host threads launching it concurrently
// with different shared-memory sizes never lower the limit under one
// another's launches.
template <class F>
inline void allow_max_dynamic_smem(F* fn) {
  static const int optin = [] {
    int d = 0, v = 0;
    cudaGetDevice(&d);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, d);
    return v;
  }();
  cudaFuncAttributes fa;
  if (cudaFuncGetAttributes(&fa, fn) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes) !=
      cudaSuccess)
    cudaGetLastError();
}
void note_cuda_error(int e);   // the CUDA error behind the last HFB_ERR_CUDA of this host thread
// Tensor map of a rows x row_floats fp32 matrix (row pitch row_floats) read in
// box_rows x 32-float boxes with the 128-byte swizzle, rows past ``rows``
// reading as zero; false when the driver's encoder is unavailable or the
// base is not 16-byte aligned.
bool encode_fp32_rows_map(CUtensorMap* m, const void* base, uint64_t row_floats, uint64_t rows, uint32_t box_rows);
void count_launch();

#define HFB_CHECK_LAUNCH()                                            \
  do {                                                                \
    hfb::count_launch();                                              \
    cudaError_t e_ = cudaGetLastError();                              \
    if (e_ != cudaSuccess) {                                          \
      hfb::note_cuda_error((int)e_);                                  \
      return HFB_ERR_CUDA;                                            \
    }                                                                 \
  } while (0)

// Supported cubic grid sizes; ``fn`` is a generic lambda taking
// std::integral_constant<int, N>.
template <class F>
int dispatch_n(int n, F&& fn) {
  switch (n) {
    case 8: return fn(std::integral_constant<int, 8>{});
    case 16: return fn(std::integral_constant<int, 16>{});
    case 24: return fn(std::integral_constant<int, 24>{});
    case 32: return fn(std::integral_constant<int, 32>{});
    case 40: return fn(std::integral_constant<int, 40>{});
    case 48: return fn(std::integral_constant<int, 48>{});
    default: return HFB_ERR_UNSUPPORTED_GRID;
  }
}

// Device-side error latch (first error wins).
__device__ __forceinline__ void latch_error(int* st, int code) { atomicCAS(st, 0, code); }

}  // namespace hfb
