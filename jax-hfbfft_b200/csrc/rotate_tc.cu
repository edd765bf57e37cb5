// Single-precision state rotation on the tcgen05 tensor cores.
//
// out1_j = sum_i psi_i U_ij and out2_j = sum_i psi_i L_ij (the rotation of
// diagstep, static.py:416-458) for complex64 states, as one real GEMM with
// both operands K-major:
//   * psi is first transposed to psiT[k][i] (k the 2 n^3 grid points of a
//     state, i the states padded to 16), so a row of A is psiT[k] with the
//     (re, im) of the states interleaved along K;
//   * B holds two rows per output j: (Re W_ij, -Im W_ij) and (Im W_ij, Re W_ij)
//     interleaved over i, so A B^T gives Re and Im of the output side by
//     side (W = U for j < ns, L for ns <= j < 2 ns);
//   * operands are split x = hi + lo (tf32) and D accumulates hi hi + hi lo
//     + lo hi, as in the Gram kernel.
// B is small (4 ns rows x 2 ns reals): it is split once, written in the
// shared-memory tile layout, and each K block of it is brought in by one
// bulk copy.  A CTA loops over tasks (128 grid points x one 144-row chunk of
// B); 7 producer warps split and store the psiT rows, one thread issues the
// MMAs into one of two TMEM accumulators per 32-real K block, and 8
// epilogue warps drain each block's accumulator into fp32 registers and
// write the finished outputs (consecutive lanes hold consecutive grid
// points, so the stores are coalesced).  Every wait is bounded; a timeout
// latches HFB_ERR_CUDA, drains the MMAs in flight and releases TMEM.
// rotate_tma_kernel (the default; HFB_TMA_FEED=0 at context creation selects
// rotate_tc_kernel) brings the psiT blocks in by TMA and splits A into
// tensor memory.
#include <math.h>
#include "hfb_ctx.cuh"
#include "tc_sm100.cuh"

namespace hfb {

namespace {

constexpr int kRtProducerWarps = 7;
constexpr int kRtEpilogueWarps = 8;
constexpr int kRtThreads = 32 * (kRtProducerWarps + 1 + kRtEpilogueWarps);
constexpr int kRtStages = 3;
constexpr int kRtN = 144;                     // B rows per chunk (72 outputs), MMA N
constexpr int kRtGroups = kRtN / 16;          // 16-column TMEM groups
constexpr int kRtMaxGroups = (kRtGroups + 1) / 2;
constexpr int kRtTmemCols = 512;
constexpr uint32_t kRtABytes = 128 * 128;     // 128 rows x 128 bytes
constexpr uint32_t kRtBBytes = kRtN * 128;    // one hi or lo B tile
constexpr uint32_t kRtStage = 2 * kRtABytes + 2 * kRtBBytes;
constexpr int kRtRowsPerPass = kRtProducerWarps * 32 / 8;
constexpr int kRtItemsA = (128 + kRtRowsPerPass - 1) / kRtRowsPerPass;
constexpr long long kRtWaitLimit = 2000000000LL;

static_assert(kRtABytes % 1024 == 0 && kRtBBytes % 1024 == 0, "tile bases must stay 1024-byte aligned");

// psiT[k][i] = psi[i][k] (i < ns), 0 for ns <= i < ldT
__global__ void psi_transpose_kernel(const float2* __restrict__ psi, float2* __restrict__ psiT, int ns, int ldT,
                                     size_t K) {
  __shared__ float2 t[32][33];
  const size_t k0 = (size_t)blockIdx.x * 32;
  const int i0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + r;
    const size_t k = k0 + threadIdx.x;
    t[r][threadIdx.x] = (i < ns && k < K) ? psi[(size_t)i * K + k] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const size_t k = k0 + r;
    const int i = i0 + threadIdx.x;
    if (k < K && i < ldT) psiT[k * ldT + i] = t[threadIdx.x][r];
  }
}

// B tiles in the shared-memory layout: for chunk c and K block kb, the hi
// tile (kRtN rows x 128 swizzled bytes) followed by the lo tile.
__global__ void rot_b_prep_kernel(const double2* __restrict__ U, const double2* __restrict__ L, int ld, int ns,
                                  int nkb, int nchunk, unsigned char* __restrict__ bt) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int total = nchunk * nkb * kRtN * 8;
  if (e >= total) return;
  const int c16 = e % 8, row = (e / 8) % kRtN, kb = (e / (8 * kRtN)) % nkb, ch = e / (8 * kRtN * nkb);
  const int R = ch * kRtN + row, j = R / 2, comp = R % 2;
  float v[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int kk = kb * 32 + c16 * 4 + q;   // real K index = 2 i + c_in
    const int i = kk / 2, cin = kk % 2;
    double2 w = make_double2(0.0, 0.0);
    if (i < ns && j < 2 * ns) w = j < ns ? U[(size_t)i * ld + j] : L[(size_t)i * ld + (j - ns)];
    double x;
    if (comp == 0) x = cin == 0 ? w.x : -w.y;
    else x = cin == 0 ? w.y : w.x;
    v[q] = (float)x;
  }
  float4 h, l;
  tc::split_tf32(v[0], h.x, l.x);
  tc::split_tf32(v[1], h.y, l.y);
  tc::split_tf32(v[2], h.z, l.z);
  tc::split_tf32(v[3], h.w, l.w);
  unsigned char* base = bt + ((size_t)ch * nkb + kb) * 2 * kRtBBytes;
  const uint32_t o = tc::sw128_offset(row, c16);
  *reinterpret_cast<float4*>(base + o) = h;
  *reinterpret_cast<float4*>(base + kRtBBytes + o) = l;
}

struct RtJob {
  size_t K;           // complex grid points per state (2 n^3)
  int ns, ldT, nkb, nchunk, ntile, ntask;
};

__global__ void __launch_bounds__(kRtThreads, 1)
rotate_tc_kernel(RtJob job, const float* __restrict__ psiT, const unsigned char* __restrict__ bt,
                 float2* __restrict__ out1, float2* __restrict__ out2, int* status) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  __shared__ uint64_t full[kRtStages], empty[kRtStages], dfull[2], dempty[2], fin;
  __shared__ uint32_t tbase;
  __shared__ volatile int abort_flag;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid & 31;
  // this CTA's tasks: blockIdx.x, blockIdx.x + gridDim.x, ...; each task is
  // nkb windows (K blocks)
  const int my_tasks = job.ntask > (int)blockIdx.x ? (job.ntask - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const int nwin = my_tasks * job.nkb;

  if (tid == 0) {
    for (int s = 0; s < kRtStages; ++s) {
      tc::mbar_init(&full[s], kRtProducerWarps + 1);
      tc::mbar_init(&empty[s], 1);
    }
    for (int d = 0; d < 2; ++d) {
      tc::mbar_init(&dfull[d], 1);
      tc::mbar_init(&dempty[d], kRtEpilogueWarps);
    }
    tc::mbar_init(&fin, 1);
    abort_flag = 0;
  }
  if (warp == kRtProducerWarps) {
    tc::tmem_alloc(&tbase, kRtTmemCols);
    tc::tmem_relinquish();
  }
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = tbase;

  auto wait = [&](uint64_t* bar, uint32_t parity) -> bool {
    if (tc::mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!tc::mbar_try_wait(bar, parity)) {
      if (abort_flag) return false;
      if (clock64() - t0 > kRtWaitLimit) {
        abort_flag = 1;
        latch_error(status, HFB_ERR_CUDA);
        return false;
      }
    }
    return true;
  };
  auto task_of = [&](int w) { return (int)blockIdx.x + (w / job.nkb) * (int)gridDim.x; };

  if (warp < kRtProducerWarps) {
    // ---------------------------------------------------------- producers
    const int c = tid & 7, r0 = tid >> 3;
    const size_t rowf = 2 * (size_t)job.ldT;   // floats per psiT row
    for (int w = 0; w < nwin; ++w) {
      const int s = w % kRtStages;
      if (w >= kRtStages && !wait(&empty[s], (uint32_t)((w / kRtStages - 1) & 1))) break;
      const int t = task_of(w), kb = w % job.nkb;
      const int tile = t / job.nchunk, ch = t % job.nchunk;
      unsigned char* st = smem + (size_t)s * kRtStage;
      if (tid == 0) {
        tc::mbar_arrive_expect_tx(&full[s], 2 * kRtBBytes);
        tc::bulk_g2s(st + 2 * kRtABytes, bt + ((size_t)ch * job.nkb + kb) * 2 * kRtBBytes, 2 * kRtBBytes, &full[s]);
      }
      const size_t off = (size_t)kb * 32 + 4 * c;
      float4 va[kRtItemsA];
#pragma unroll
      for (int i = 0; i < kRtItemsA; ++i) {
        const int rl = r0 + kRtRowsPerPass * i;
        const size_t k = (size_t)tile * 128 + rl;
        if (rl < 128 && k < job.K) va[i] = __ldg(reinterpret_cast<const float4*>(psiT + k * rowf + off));
        else va[i] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
#pragma unroll
      for (int i = 0; i < kRtItemsA; ++i) {
        const int rl = r0 + kRtRowsPerPass * i;
        if (rl >= 128) continue;
        const float4 v = va[i];
        float4 h, l;
        tc::split_tf32(v.x, h.x, l.x);
        tc::split_tf32(v.y, h.y, l.y);
        tc::split_tf32(v.z, h.z, l.z);
        tc::split_tf32(v.w, h.w, l.w);
        const uint32_t o = tc::sw128_offset(rl, c);
        *reinterpret_cast<float4*>(st + o) = h;
        *reinterpret_cast<float4*>(st + kRtABytes + o) = l;
      }
      tc::fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&full[s]);
    }
  } else if (warp == kRtProducerWarps) {
    // ---------------------------------------------------------------- MMA
    if (lane == 0) {
      const uint32_t idesc = tc::idesc_tf32(128, kRtN);
      for (int w = 0; w < nwin; ++w) {
        const int s = w % kRtStages, d = w & 1;
        if (!wait(&full[s], (uint32_t)((w / kRtStages) & 1))) break;
        if (w >= 2 && !wait(&dempty[d], (uint32_t)((w / 2 - 1) & 1))) break;
        tc::fence_after();
        const uint32_t sa = tc::smem_u32(smem + (size_t)s * kRtStage);
        const uint32_t ahi = sa, alo = sa + kRtABytes, bhi = sa + 2 * kRtABytes, blo = bhi + kRtBBytes;
        const uint32_t dt = tmem + (uint32_t)(d * 256);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          tc::mma_tf32(dt, tc::sw128_desc(ahi + 32 * k), tc::sw128_desc(bhi + 32 * k), idesc, k > 0);
          tc::mma_tf32(dt, tc::sw128_desc(ahi + 32 * k), tc::sw128_desc(blo + 32 * k), idesc, 1);
          tc::mma_tf32(dt, tc::sw128_desc(alo + 32 * k), tc::sw128_desc(bhi + 32 * k), idesc, 1);
        }
        tc::mma_commit(&empty[s]);
        tc::mma_commit(&dfull[d]);
      }
      tc::mma_commit(&fin);
      if (!tc::mbar_wait(&fin, 0, kRtWaitLimit)) latch_error(status, HFB_ERR_CUDA);
    }
    __syncwarp();
  } else {
    // ----------------------------------------------------------- epilogue
    const int q = warp & 3;
    const int half = (warp - kRtProducerWarps - 1) / 4;
    const int gbeg = half ? kRtMaxGroups : 0, gcnt = half ? kRtGroups - kRtMaxGroups : kRtMaxGroups;
    float acc[kRtMaxGroups][16];
#pragma unroll
    for (int g = 0; g < kRtMaxGroups; ++g)
#pragma unroll
      for (int i = 0; i < 16; ++i) acc[g][i] = 0.f;
    for (int w = 0; w < nwin; ++w) {
      const int d = w & 1;
      if (!wait(&dfull[d], (uint32_t)((w / 2) & 1))) break;
      tc::fence_after();
      const uint32_t ta = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(d * 256);
#pragma unroll
      for (int g = 0; g < kRtMaxGroups; ++g) {
        if (g < gcnt) {
          float v[16];
          tc::tmem_ld16(ta + (uint32_t)((gbeg + g) * 16), v);
#pragma unroll
          for (int i = 0; i < 16; ++i) acc[g][i] += v[i];
        }
      }
      tc::fence_before();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&dempty[d]);
      if (w % job.nkb == job.nkb - 1) {
        // last K block of the task: outputs (re, im) at columns (2 m, 2 m + 1)
        const int t = task_of(w);
        const int tile = t / job.nchunk, ch = t % job.nchunk;
        const size_t k = (size_t)tile * 128 + q * 32 + lane;
#pragma unroll
        for (int g = 0; g < kRtMaxGroups; ++g) {
          if (g < gcnt) {
#pragma unroll
            for (int i = 0; i < 16; i += 2) {
              const int j = (ch * kRtN + (gbeg + g) * 16 + i) / 2;
              if (k < job.K && !abort_flag) {
                const float2 v = make_float2(acc[g][i], acc[g][i + 1]);
                if (j < job.ns) out1[(size_t)j * job.K + k] = v;
                else if (j < 2 * job.ns) out2[(size_t)(j - job.ns) * job.K + k] = v;
              }
              acc[g][i] = 0.f;
              acc[g][i + 1] = 0.f;
            }
          }
        }
      }
    }
  }
  tc::fence_before();
  __syncthreads();
  if (warp == kRtProducerWarps) {
    tc::fence_after();
    tc::tmem_dealloc(tmem, kRtTmemCols);
  }
}

// The same rotation with the psiT K blocks brought in by the tensor-memory
// accelerator (one 128-row x 32-float swizzled box per K block, beside the
// bulk copy of the B tiles) and A split into tensor memory:
//   warp 0      (one thread) TMA + bulk copy into a 3-stage ring;
//   warp 1      (one thread) MMAs with A from TMEM; owns the TMEM allocation;
//   warps 4-7   split A (one row per thread) into the stage's 64 TMEM columns;
//   warps 8-15  drain and store as in rotate_tc_kernel.
// TMEM: accumulators at columns 0 and 160, A stages at 320 + 64 s.
constexpr uint32_t kRqRawA = 128 * 128;
constexpr uint32_t kRqStage = kRqRawA + 2 * kRtBBytes;
constexpr int kRqConvWarps = 4;
constexpr uint32_t kRqD1 = 160, kRqACol = 320;

__global__ void __launch_bounds__(kRtThreads, 1)
rotate_tma_kernel(RtJob job, const __grid_constant__ CUtensorMap mpt, const unsigned char* __restrict__ bt,
                  float2* __restrict__ out1, float2* __restrict__ out2, int* status, long long limit) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  __shared__ uint64_t raw_full[kRtStages], empty[kRtStages], conv_full[kRtStages], dfull[2], dempty[2], fin;
  __shared__ uint32_t tbase;
  __shared__ volatile int abort_flag;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid & 31;
  const int my_tasks = job.ntask > (int)blockIdx.x ? (job.ntask - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const int nwin = my_tasks * job.nkb;

  if (tid == 0) {
    for (int s = 0; s < kRtStages; ++s) {
      tc::mbar_init(&raw_full[s], 1);
      tc::mbar_init(&empty[s], 1);
      tc::mbar_init(&conv_full[s], kRqConvWarps);
    }
    for (int d = 0; d < 2; ++d) {
      tc::mbar_init(&dfull[d], 1);
      tc::mbar_init(&dempty[d], kRtEpilogueWarps);
    }
    tc::mbar_init(&fin, 1);
    abort_flag = 0;
  }
  if (warp == 1) {
    tc::tmem_alloc(&tbase, kRtTmemCols);
    tc::tmem_relinquish();
  }
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = tbase;

  auto wait = [&](uint64_t* bar, uint32_t parity) -> bool {
    if (tc::mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!tc::mbar_try_wait(bar, parity)) {
      if (abort_flag) return false;
      if (clock64() - t0 > limit) {
        abort_flag = 1;
        latch_error(status, HFB_ERR_CUDA);
        return false;
      }
    }
    return true;
  };
  auto task_of = [&](int w) { return (int)blockIdx.x + (w / job.nkb) * (int)gridDim.x; };

  if (warp == 0) {
    // ------------------------------------------------------- TMA and bulk
    if (lane == 0) {
      int issued = 0;
      for (int w = 0; w < nwin; ++w) {
        const int s = w % kRtStages;
        if (w >= kRtStages && !wait(&empty[s], (uint32_t)((w / kRtStages - 1) & 1))) break;
        const int t = task_of(w), kb = w % job.nkb;
        const int tile = t / job.nchunk, ch = t % job.nchunk;
        unsigned char* st = smem + (size_t)s * kRqStage;
        tc::mbar_arrive_expect_tx(&raw_full[s], kRqRawA + 2 * kRtBBytes);
        tc::tma_load_2d(st, &mpt, kb * 32, tile * 128, &raw_full[s]);
        tc::bulk_g2s(st + kRqRawA, bt + ((size_t)ch * job.nkb + kb) * 2 * kRtBBytes, 2 * kRtBBytes, &raw_full[s]);
        issued = w + 1;
      }
      for (int w = max(0, issued - kRtStages); w < issued; ++w)
        if (!tc::mbar_wait(&raw_full[w % kRtStages], (uint32_t)((w / kRtStages) & 1), limit))
          latch_error(status, HFB_ERR_CUDA);
    }
    __syncwarp();
  } else if (warp == 1) {
    // ---------------------------------------------------------------- MMA
    if (lane == 0) {
      const uint32_t idesc = tc::idesc_tf32(128, kRtN);
      for (int w = 0; w < nwin; ++w) {
        const int s = w % kRtStages, d = w & 1;
        if (!wait(&conv_full[s], (uint32_t)((w / kRtStages) & 1))) break;
        if (w >= 2 && !wait(&dempty[d], (uint32_t)((w / 2 - 1) & 1))) break;
        tc::fence_after();
        const uint32_t bhi = tc::smem_u32(smem + (size_t)s * kRqStage + kRqRawA), blo = bhi + kRtBBytes;
        const uint32_t dt = tmem + (uint32_t)d * kRqD1, at = tmem + kRqACol + (uint32_t)s * 64;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          tc::mma_tf32_ta(dt, at + 8 * k, tc::sw128_desc(bhi + 32 * k), idesc, k > 0);
          tc::mma_tf32_ta(dt, at + 8 * k, tc::sw128_desc(blo + 32 * k), idesc, 1);
          tc::mma_tf32_ta(dt, at + 32 + 8 * k, tc::sw128_desc(bhi + 32 * k), idesc, 1);
        }
        tc::mma_commit(&empty[s]);
        tc::mma_commit(&dfull[d]);
      }
      tc::mma_commit(&fin);
      if (!tc::mbar_wait(&fin, 0, limit)) latch_error(status, HFB_ERR_CUDA);
    }
    __syncwarp();
  } else if (warp >= 4 && warp < 8) {
    // ------------------------------------------------------- A converters
    const int q = warp & 3, r = 32 * q + lane;
    for (int w = 0; w < nwin; ++w) {
      const int s = w % kRtStages;
      if (!wait(&raw_full[s], (uint32_t)((w / kRtStages) & 1))) break;
      const unsigned char* st = smem + (size_t)s * kRqStage;
      const uint32_t ta = tmem + ((uint32_t)(q * 32) << 16) + kRqACol + (uint32_t)s * 64;
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        float hv[16], lv[16];
#pragma unroll
        for (int c4 = 0; c4 < 4; ++c4) {
          const float4 v = *reinterpret_cast<const float4*>(st + tc::sw128_offset(r, 4 * half + c4));
          const float x4[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            tc::split_tf32(x4[i], hv[4 * c4 + i], lv[4 * c4 + i]);
          }
        }
        tc::tmem_st16(ta + 16 * half, hv);
        tc::tmem_st16(ta + 32 + 16 * half, lv);
      }
      tc::tmem_st_wait();
      tc::fence_before();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&conv_full[s]);
    }
  } else if (warp >= 8) {
    // ----------------------------------------------------------- epilogue
    const int q = warp & 3;
    const int half = (warp - 8) / 4;
    const int gbeg = half ? kRtMaxGroups : 0, gcnt = half ? kRtGroups - kRtMaxGroups : kRtMaxGroups;
    float acc[kRtMaxGroups][16];
#pragma unroll
    for (int g = 0; g < kRtMaxGroups; ++g)
#pragma unroll
      for (int i = 0; i < 16; ++i) acc[g][i] = 0.f;
    for (int w = 0; w < nwin; ++w) {
      const int d = w & 1;
      if (!wait(&dfull[d], (uint32_t)((w / 2) & 1))) break;
      tc::fence_after();
      const uint32_t ta = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)d * kRqD1;
#pragma unroll
      for (int g = 0; g < kRtMaxGroups; ++g) {
        if (g < gcnt) {
          float v[16];
          tc::tmem_ld16(ta + (uint32_t)((gbeg + g) * 16), v);
#pragma unroll
          for (int i = 0; i < 16; ++i) acc[g][i] += v[i];
        }
      }
      tc::fence_before();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&dempty[d]);
      if (w % job.nkb == job.nkb - 1) {
        const int t = task_of(w);
        const int tile = t / job.nchunk, ch = t % job.nchunk;
        const size_t k = (size_t)tile * 128 + q * 32 + lane;
#pragma unroll
        for (int g = 0; g < kRtMaxGroups; ++g) {
          if (g < gcnt) {
#pragma unroll
            for (int i = 0; i < 16; i += 2) {
              const int j = (ch * kRtN + (gbeg + g) * 16 + i) / 2;
              if (k < job.K && !abort_flag) {
                const float2 v = make_float2(acc[g][i], acc[g][i + 1]);
                if (j < job.ns) out1[(size_t)j * job.K + k] = v;
                else if (j < 2 * job.ns) out2[(size_t)(j - job.ns) * job.K + k] = v;
              }
              acc[g][i] = 0.f;
              acc[g][i + 1] = 0.f;
            }
          }
        }
      }
    }
  }
  tc::fence_before();
  __syncthreads();
  if (warp == 1) {
    tc::fence_after();
    tc::tmem_dealloc(tmem, kRtTmemCols);
  }
}

}  // namespace

static RtJob rt_job(hfb_ctx_s* c, int ns) {
  RtJob job{};
  job.K = (size_t)2 * c->n * c->n * c->n;
  job.ns = ns;
  job.ldT = (ns + 15) / 16 * 16;
  job.nkb = job.ldT / 16;
  job.nchunk = (4 * ns + kRtN - 1) / kRtN;
  job.ntile = (int)(job.K / 128);
  job.ntask = job.ntile * job.nchunk;
  return job;
}

// The job's buffer (psiT, then the B tiles) in scratch slot ``slot``.
static unsigned char* rt_buffer(hfb_ctx_s* c, const RtJob& job, int slot, size_t* tbytes) {
  *tbytes = sizeof(float2) * job.K * (size_t)job.ldT;
  const size_t bbytes = (size_t)job.nchunk * job.nkb * 2 * kRtBBytes;
  return (unsigned char*)scratch(c, slot, *tbytes + bbytes + 1024);
}

// psiT (the K-major A operand) of ns complex64 states at psi, into the
// buffer of rotation ``which`` (0 or 1): the transpose depends on psi only,
// so the diagonalisation step issues it early, beside the Gram and the
// eigensolve.  HFB_ERR_UNSUPPORTED_GRID as rotate_tc_launch.
int rotate_tc_transpose(hfb_ctx_s* c, int which, int ns, const void* psi, cudaStream_t st) {
  if (ns <= 0) return HFB_OK;
  const RtJob job = rt_job(c, ns);
  if (job.K % 128 != 0) return HFB_ERR_UNSUPPORTED_GRID;
  size_t tbytes;
  unsigned char* buf = rt_buffer(c, job, which ? hfb_ctx_s::S_ROT2 : hfb_ctx_s::S_ROT, &tbytes);
  if (!buf) return HFB_ERR_ALLOC;
  dim3 tg((unsigned)((job.K + 31) / 32), (unsigned)((job.ldT + 31) / 32));
  psi_transpose_kernel<<<tg, dim3(32, 8), 0, st>>>((const float2*)psi, (float2*)buf, ns, job.ldT, job.K);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

// out1 = psi U, out2 = psi L for ns complex64 states at psi (offset already
// applied).  ``pre`` = 0 or 1: psiT is already in the buffer of that
// rotation (rotate_tc_transpose on the same states); -1: transposed here.
// HFB_ERR_UNSUPPORTED_GRID when the grid's 2 n^3 is not a multiple of 128
// (the caller then uses the CUDA-core kernel).
int rotate_tc_launch(hfb_ctx_s* c, int ns, const void* psi, const double2* U, const double2* L, int ld, void* out1,
                     void* out2, cudaStream_t st, int pre) {
  if (ns <= 0) return HFB_OK;
  const RtJob job = rt_job(c, ns);
  const size_t K = job.K;
  if (K % 128 != 0) return HFB_ERR_UNSUPPORTED_GRID;
  size_t tbytes;
  unsigned char* buf = rt_buffer(c, job, pre == 1 ? hfb_ctx_s::S_ROT2 : hfb_ctx_s::S_ROT, &tbytes);
  if (!buf) return HFB_ERR_ALLOC;
  float2* psiT = (float2*)buf;
  unsigned char* bt = buf + ((tbytes + 1023) / 1024) * 1024;
  if (pre < 0) {
    dim3 tg((unsigned)((K + 31) / 32), (unsigned)((job.ldT + 31) / 32));
    psi_transpose_kernel<<<tg, dim3(32, 8), 0, st>>>((const float2*)psi, psiT, ns, job.ldT, K);
    HFB_CHECK_LAUNCH();
  }
  const int nprep = job.nchunk * job.nkb * kRtN * 8;
  rot_b_prep_kernel<<<(nprep + 255) / 256, 256, 0, st>>>(U, L, ld, ns, job.nkb, job.nchunk, bt);
  HFB_CHECK_LAUNCH();
  int nsm = 148;
  {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  }
  const int grid = job.ntask < nsm ? job.ntask : nsm;
  CUtensorMap mpt;
  if (c->tma_feed && encode_fp32_rows_map(&mpt, psiT, 2 * (uint64_t)job.ldT, K, 128)) {
    const size_t smem = 1024 + (size_t)kRtStages * kRqStage;
    allow_max_dynamic_smem(rotate_tma_kernel);
    rotate_tma_kernel<<<grid, kRtThreads, smem, st>>>(job, mpt, bt, (float2*)out1, (float2*)out2, c->dev_status,
                                                      c->wait_limit);
  } else {
    const size_t smem = 1024 + (size_t)kRtStages * kRtStage;
    allow_max_dynamic_smem(rotate_tc_kernel);
    rotate_tc_kernel<<<grid, kRtThreads, smem, st>>>(job, (const float*)psiT, bt, (float2*)out1, (float2*)out2,
                                                     c->dev_status);
  }
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

}  // namespace hfb
