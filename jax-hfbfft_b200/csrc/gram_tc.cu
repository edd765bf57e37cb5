// Single-precision Gram matrices on the tcgen05 tensor cores.
//
// C_a = wxyz Psi^H X_a (X = psi, hampsi, hmfpsi, v_pair psi; static.py:
// 283-290, 380-387 and construct_hfb_matrices 484-577) for complex64 states.
// The complex product is written as one real GEMM over the interleaved
// (re, im) storage: with A' = [Psi ; Psi~] (Psi~ row = (-im, re) per
// element), D = A' X^T gives Re C in rows 0..n-1 and Im C in rows n..2n-1.
// Operands are split as x = hi + lo with hi = tf32(x), lo = x - hi (exact,
// left unrounded: the MMA takes its tf32 part) and D accumulates hi*hi +
// hi*lo + lo*hi (the three-term tf32 scheme, about 21 significant bits per
// product).
//
// One CTA owns one 128-row block of A' for one matrix and one slice of K.
// (Feeding the K blocks by TMA, with A split into tensor memory as the
// rotation does, measured slower here: 2.9-3.2 ms against 2.0 ms for the
// 140 Pb208 neutron states, with 8-row or 128-row boxes and with a deeper
// raw ring; the split of B then sits on six warps instead of seven, four
// of which also split A.)
//   warps 0-6   load a 32-float K block of the rows from global memory,
//               split it and store it into a 128-byte-swizzled stage
//               (3-stage ring);
//   warp 7      issues the MMAs (M = 128, N = n padded to 16, K = 8) into
//               one of two TMEM accumulators, which starts from zero every
//               four K blocks;
//   warps 8-15  drain the finished accumulator into fp32 registers every
//               four K blocks, so the tensor core's own fp32 accumulation
//               spans at most 48 MMAs and the sum over drains is rounded to
//               nearest.
// Per-slice partial sums are added in fp64 in a fixed order by a second
// kernel, which also scatters Re/Im rows into the complex outputs.
// Every wait is bounded; a timeout latches HFB_ERR_CUDA, drains the MMAs
// in flight and releases TMEM before returning.
#include <math.h>
#include "hfb_ctx.cuh"
#include "tc_sm100.cuh"

namespace hfb {

namespace {

constexpr int kTcProducerWarps = 7;   // 16 warps in all: 4 per SM sub-partition, 128 registers each
constexpr int kTcEpilogueWarps = 8;
constexpr int kTcThreads = 32 * (kTcProducerWarps + 1 + kTcEpilogueWarps);
constexpr int kTcStages = 3;
constexpr int kTcMaxNp = 160;           // padded states per block handled here
constexpr int kTcMaxGroups = 5;         // 16-column groups per epilogue thread
constexpr int kTcMaxUnits = 32;
constexpr int kTcRowsPerPass = kTcProducerWarps * 32 / 8;   // 8 threads per 128-byte row
constexpr int kTcItemsA = (128 + kTcRowsPerPass - 1) / kTcRowsPerPass;
constexpr int kTcItemsB = (kTcMaxNp + kTcRowsPerPass - 1) / kTcRowsPerPass;
constexpr int kTcTmemCols = 512;        // two accumulators at columns 0 and 256
constexpr uint32_t kTcABytes = 128 * 128;   // 128 rows x 128 bytes
constexpr long long kTcWaitLimit = 2000000000LL;
// K blocks accumulated in TMEM between drains into registers: 4 measured
// 6 % faster than 1 on Pb208 (1.96 ms against 2.09 ms for the 140 neutron
// states) and stays inside the 3e-6 bar of the single-precision Gram test
constexpr int kTcDrain = 4;

struct TcUnit {
  unsigned char b, a, mb, pad;
};
struct TcJob {
  int nunit, kchunks, kb_total, n3;
  int drain;                      // K blocks accumulated in TMEM between drains
  TcUnit u[kTcMaxUnits];
  int s0[2], ns[2], np[2];
  const double* vp[2];
  signed char unit_of[2][4][4];   // [block][matrix][m-block] -> unit
};

__device__ __forceinline__ uint32_t stage_bytes(int np) { return 2 * kTcABytes + 2 * (uint32_t)np * 128; }

__global__ void __launch_bounds__(kTcThreads, 1)
gram_tc_kernel(TcJob job, const float* __restrict__ psi, const float* __restrict__ hampsi,
               const float* __restrict__ hmfpsi, float* __restrict__ part, int* status) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  __shared__ uint64_t full[kTcStages], empty[kTcStages], dfull[2], dempty[2], fin;
  __shared__ uint32_t tbase;
  __shared__ volatile int abort_flag;

  const int unit = blockIdx.x % job.nunit, chunk = blockIdx.x / job.nunit;
  const TcUnit U = job.u[unit];
  const int b = U.b, am = U.a, mb = U.mb;
  const int n = job.ns[b], np = job.np[b];
  const size_t K = 2 * (size_t)job.n3;                 // complex elements per state
  const int kb0 = (int)((long long)job.kb_total * chunk / job.kchunks);
  const int kb1 = (int)((long long)job.kb_total * (chunk + 1) / job.kchunks);
  const int nwin = kb1 - kb0;
  const uint32_t sbytes = stage_bytes(np);
  const int tid = threadIdx.x, warp = tid / 32, lane = tid & 31;

  if (tid == 0) {
    for (int s = 0; s < kTcStages; ++s) {
      tc::mbar_init(&full[s], kTcProducerWarps);
      tc::mbar_init(&empty[s], 1);
    }
    for (int d = 0; d < 2; ++d) {
      tc::mbar_init(&dfull[d], 1);
      tc::mbar_init(&dempty[d], kTcEpilogueWarps);
    }
    tc::mbar_init(&fin, 1);
    abort_flag = 0;
  }
  if (warp == kTcProducerWarps) {
    tc::tmem_alloc(&tbase, kTcTmemCols);
    tc::tmem_relinquish();
  }
  // zero every stage once: padding rows are never written again
  for (uint32_t e = tid; e < kTcStages * sbytes / 16; e += blockDim.x)
    reinterpret_cast<float4*>(smem)[e] = make_float4(0.f, 0.f, 0.f, 0.f);
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
      if (clock64() - t0 > kTcWaitLimit) {
        abort_flag = 1;
        latch_error(status, HFB_ERR_CUDA);
        return false;
      }
    }
    return true;
  };

  if (warp < kTcProducerWarps) {
    // ---------------------------------------------------------- producers
    const int c = tid & 7;            // 16-byte chunk of the 128-byte row
    const int r0 = tid >> 3;          // first row; rows r0 + kTcRowsPerPass i
    const size_t rowf = 2 * K;        // floats per state
    // A' rows: state index (or -1) and whether the row is Psi~
    int rowA[kTcItemsA];
    unsigned tmask = 0;
#pragma unroll
    for (int i = 0; i < kTcItemsA; ++i) {
      const int rl = r0 + kTcRowsPerPass * i, rg = mb * 128 + rl;
      rowA[i] = rl >= 128 ? -1 : rg < n ? rg : (rg < 2 * n ? rg - n : -1);
      if (rg >= n && rg < 2 * n) tmask |= 1u << i;
    }
    const float* pa = psi + (size_t)job.s0[b] * rowf;
    const float* pb = (am == 1 ? hampsi : am == 2 ? hmfpsi : psi) + (size_t)job.s0[b] * rowf;
    const double* vp = job.vp[b];
    for (int w = 0; w < nwin; ++w) {
      const int s = w % kTcStages;
      if (w >= kTcStages && !wait(&empty[s], (uint32_t)((w / kTcStages - 1) & 1))) break;
      const size_t off = (size_t)(kb0 + w) * 32 + 4 * c;
      float4 va[kTcItemsA], vb[kTcItemsB];
#pragma unroll
      for (int i = 0; i < kTcItemsA; ++i)
        if (rowA[i] >= 0) va[i] = __ldg(reinterpret_cast<const float4*>(pa + (size_t)rowA[i] * rowf + off));
#pragma unroll
      for (int i = 0; i < kTcItemsB; ++i) {
        const int j = r0 + kTcRowsPerPass * i;
        if (j < n) vb[i] = __ldg(reinterpret_cast<const float4*>(pb + (size_t)j * rowf + off));
      }
      float v0 = 1.f, v1 = 1.f;
      if (am == 3) {
        const size_t k = (off / 2) % (size_t)job.n3;
        v0 = (float)vp[k];
        v1 = (float)vp[k + 1];
      }
      unsigned char* st = smem + (size_t)s * sbytes;
      auto put = [&](unsigned char* hi_base, uint32_t lo_delta, int row, float4 v) {
        float4 h, l;
        tc::split_tf32(v.x, h.x, l.x);
        tc::split_tf32(v.y, h.y, l.y);
        tc::split_tf32(v.z, h.z, l.z);
        tc::split_tf32(v.w, h.w, l.w);
        const uint32_t o = tc::sw128_offset(row, c);
        *reinterpret_cast<float4*>(hi_base + o) = h;
        *reinterpret_cast<float4*>(hi_base + lo_delta + o) = l;
      };
#pragma unroll
      for (int i = 0; i < kTcItemsA; ++i) {
        if (rowA[i] < 0) continue;
        float4 v = va[i];
        if ((tmask >> i) & 1) v = make_float4(-v.y, v.x, -v.w, v.z);
        put(st, kTcABytes, r0 + kTcRowsPerPass * i, v);
      }
#pragma unroll
      for (int i = 0; i < kTcItemsB; ++i) {
        const int j = r0 + kTcRowsPerPass * i;
        if (j >= n) continue;
        float4 v = vb[i];
        if (am == 3) v = make_float4(v0 * v.x, v0 * v.y, v1 * v.z, v1 * v.w);
        put(st + 2 * kTcABytes, (uint32_t)np * 128, j, v);
      }
      tc::fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&full[s]);
    }
  } else if (warp == kTcProducerWarps) {
    // ---------------------------------------------------------------- MMA
    if (lane == 0) {
      const uint32_t idesc = tc::idesc_tf32(128, np);
      for (int w = 0; w < nwin; ++w) {
        const int s = w % kTcStages, e = w / job.drain, d = e & 1;
        const bool first = w % job.drain == 0, last = w % job.drain == job.drain - 1 || w == nwin - 1;
        if (!wait(&full[s], (uint32_t)((w / kTcStages) & 1))) break;
        if (first && e >= 2 && !wait(&dempty[d], (uint32_t)((e / 2 - 1) & 1))) break;
        tc::fence_after();
        const uint32_t sa = tc::smem_u32(smem + (size_t)s * sbytes);
        const uint32_t ahi = sa, alo = sa + kTcABytes, bhi = sa + 2 * kTcABytes, blo = bhi + (uint32_t)np * 128;
        const uint32_t dt = tmem + (uint32_t)(d * 256);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          tc::mma_tf32(dt, tc::sw128_desc(ahi + 32 * k), tc::sw128_desc(bhi + 32 * k), idesc, k > 0 || !first);
          tc::mma_tf32(dt, tc::sw128_desc(ahi + 32 * k), tc::sw128_desc(blo + 32 * k), idesc, 1);
          tc::mma_tf32(dt, tc::sw128_desc(alo + 32 * k), tc::sw128_desc(bhi + 32 * k), idesc, 1);
        }
        tc::mma_commit(&empty[s]);
        if (last) tc::mma_commit(&dfull[d]);
      }
      // every MMA issued above has completed once this arrives
      tc::mma_commit(&fin);
      if (!tc::mbar_wait(&fin, 0, kTcWaitLimit)) latch_error(status, HFB_ERR_CUDA);
    }
    __syncwarp();
  } else {
    // ----------------------------------------------------------- epilogue
    const int q = warp & 3;                       // TMEM lane quarter of this warp
    const int half = (warp - kTcProducerWarps - 1) / 4;   // two warps per quarter split the columns
    const int ng = np / 16, g0 = (ng + 1) / 2;
    const int gbeg = half ? g0 : 0, gcnt = half ? ng - g0 : g0;
    float acc[kTcMaxGroups][16];
#pragma unroll
    for (int g = 0; g < kTcMaxGroups; ++g)
#pragma unroll
      for (int i = 0; i < 16; ++i) acc[g][i] = 0.f;
    bool ok = true;
    const int nep = (nwin + job.drain - 1) / job.drain;
    for (int e = 0; e < nep; ++e) {
      const int d = e & 1;
      if (!wait(&dfull[d], (uint32_t)((e / 2) & 1))) { ok = false; break; }
      tc::fence_after();
      const uint32_t ta = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(d * 256);
      // two groups per load where possible: fewer load-wait round trips
#pragma unroll
      for (int g = 0; g < kTcMaxGroups; g += 2) {
        if (g + 1 < gcnt) {
          float v[32];
          tc::tmem_ld32(ta + (uint32_t)((gbeg + g) * 16), v);
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            acc[g][i] += v[i];
            acc[g + 1][i] += v[16 + i];
          }
        } else if (g < gcnt) {
          float v[16];
          tc::tmem_ld16(ta + (uint32_t)((gbeg + g) * 16), v);
#pragma unroll
          for (int i = 0; i < 16; ++i) acc[g][i] += v[i];
        }
      }
      tc::fence_before();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&dempty[d]);
    }
    if (ok && !abort_flag) {
      const int row = q * 32 + lane;
      float* o = part + ((size_t)blockIdx.x * 128 + row) * kTcMaxNp;
#pragma unroll
      for (int g = 0; g < kTcMaxGroups; ++g)
        if (g < gcnt) {
#pragma unroll
          for (int i = 0; i < 16; i += 4)
            *reinterpret_cast<float4*>(o + (gbeg + g) * 16 + i) =
                make_float4(acc[g][i], acc[g][i + 1], acc[g][i + 2], acc[g][i + 3]);
        }
    }
  }
  tc::fence_before();
  __syncthreads();
  if (warp == kTcProducerWarps) {
    tc::fence_after();
    tc::tmem_dealloc(tmem, kTcTmemCols);
  }
}

struct TcOut {
  double2* p[8];   // [block * 4 + matrix]
};

// out_a[b][i][j] = wxyz * (Re, Im) from rows i and n + i of A' X^T, the
// K slices summed in fp64 in order; Hermitian matrices mirror the upper
// triangle.
__global__ void gram_tc_reduce_kernel(TcJob job, const float* __restrict__ part, double scale, TcOut outs, int ldo,
                                      int bq, int aq) {
  const int b = bq, am = aq;
  const int n = job.ns[b];
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n * n) return;
  const int i = e / n, j = e % n;
  const bool herm = am != 1;
  if (herm && i > j) return;
  const int rre = i, rim = n + i;
  const int ure = job.unit_of[b][am][rre / 128], uim = job.unit_of[b][am][rim / 128];
  double re = 0.0, im = 0.0;
  for (int c = 0; c < job.kchunks; ++c) {
    re += (double)part[(((size_t)c * job.nunit + ure) * 128 + (rre % 128)) * kTcMaxNp + j];
    im += (double)part[(((size_t)c * job.nunit + uim) * 128 + (rim % 128)) * kTcMaxNp + j];
  }
  double2* out = outs.p[b * 4 + am];
  out[(size_t)i * ldo + j] = make_double2(scale * re, scale * im);
  if (herm && i != j) out[(size_t)j * ldo + i] = make_double2(scale * re, -scale * im);
}

}  // namespace

// Returns HFB_ERR_UNSUPPORTED_GRID when a block exceeds kTcMaxNp states
// (the caller then uses the CUDA-core kernel).
int gram_tc_launch(hfb_ctx_s* c, int nblk, const int* s0, const int* ns, const int* masks, const void* psi,
                   const void* hampsi, const void* hmfpsi, const double* const* vp, double wxyz,
                   double2* const* outs_host, int ldo, cudaStream_t st) {
  TcJob job{};
  job.n3 = c->n * c->n * c->n;
  job.kb_total = (int)(4 * (size_t)job.n3 / 32);
  for (int b = 0; b < 2; ++b)
    for (int a = 0; a < 4; ++a)
      for (int m = 0; m < 4; ++m) job.unit_of[b][a][m] = -1;
  for (int b = 0; b < nblk; ++b) {
    if (ns[b] <= 0) continue;
    job.s0[b] = s0[b];
    job.ns[b] = ns[b];
    job.np[b] = (ns[b] + 15) / 16 * 16;
    job.vp[b] = vp ? vp[b] : nullptr;
    if (job.np[b] > kTcMaxNp) return HFB_ERR_UNSUPPORTED_GRID;
    const int nmb = (2 * ns[b] + 127) / 128;
    for (int a = 0; a < 4; ++a) {
      if (!(masks[b] & (1 << a))) continue;
      for (int m = 0; m < nmb; ++m) {
        if (job.nunit >= kTcMaxUnits) return HFB_ERR_UNSUPPORTED_GRID;
        job.unit_of[b][a][m] = (signed char)job.nunit;
        job.u[job.nunit++] = TcUnit{(unsigned char)b, (unsigned char)a, (unsigned char)m, 0};
      }
    }
  }
  if (job.nunit == 0) return HFB_OK;
  // about one wave of single-CTA SMs
  int nsm = 148;
  {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  }
  job.drain = kTcDrain;
  job.kchunks = nsm / job.nunit;
  if (job.kchunks < 1) job.kchunks = 1;
  if (job.kchunks > job.kb_total) job.kchunks = job.kb_total;
  const int ncta = job.nunit * job.kchunks;
  float* part = (float*)scratch(c, hfb_ctx_s::S_GRAM, sizeof(float) * (size_t)ncta * 128 * kTcMaxNp);
  if (!part) return HFB_ERR_ALLOC;
  int npmax = 16;
  for (int b = 0; b < nblk; ++b) npmax = job.np[b] > npmax ? job.np[b] : npmax;
  const size_t smem = 1024 + (size_t)kTcStages * (2 * kTcABytes + 2 * (size_t)npmax * 128);
  allow_max_dynamic_smem(gram_tc_kernel);
  gram_tc_kernel<<<ncta, kTcThreads, smem, st>>>(job, (const float*)psi, (const float*)hampsi,
                                                 (const float*)hmfpsi, part, c->dev_status);
  HFB_CHECK_LAUNCH();
  TcOut ot;
  for (int q = 0; q < 8; ++q) ot.p[q] = outs_host[q];
  for (int b = 0; b < nblk; ++b)
    for (int a = 0; a < 4; ++a) {
      if (ns[b] <= 0 || !(masks[b] & (1 << a))) continue;
      const int nn = ns[b] * ns[b];
      gram_tc_reduce_kernel<<<(nn + 255) / 256, 256, 0, st>>>(job, part, wxyz, ot, ldo, b, a);
      HFB_CHECK_LAUNCH();
    }
  return HFB_OK;
}

}  // namespace hfb
