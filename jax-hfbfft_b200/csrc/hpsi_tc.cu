// Single-precision hpsi (hpsi01, meanfield.py:41-159) on the tcgen05 tensor
// cores.
//
// Along each axis d the derivative terms of h_q are (as in hpsi.cu)
//     out_d = L_d(D psi) + D (L_d psi - B D psi) + Nyquist term,
// with D the periodic spectral first derivative along d whose k = 0 and
// n/2 bins are zero (cderv of levels.py), B the effective mass and L_d the
// pointwise 2x2 complex current / spin-orbit operator of that axis
// (meanfield.py:63-141).  D is a real n x n matrix, so D on every line of
// a state along d is a real GEMM with K = n: the FFT path's two forward and
// two inverse line transforms per component and axis become two GEMMs.
// The Nyquist term, (pi/d)^2 mean_line(B) (-1)^j sum_l (-1)^l psi_l / n,
// takes its alternating sum from an extra output row of the first GEMM.
//
// A tile is 32 lines of one axis of one state with 4 real parts each
// (Re / Im of the two spinor components): 128 GEMM rows, row = 4 line +
// part, so the 4 parts of a grid point sit in 4 adjacent lanes.
//   staging    each thread (row, every other 8-point chunk) reads psi, computes
//              n = L_d psi (kept in spare TMEM columns) and for the z pass
//              the local upot / spin terms (stored into the second
//              accumulator), splits psi = hi + lo (tf32) and stores both
//              into TMEM, where tcgen05.mma reads its A operand;
//   GEMM 1     e = D psi and the alternating sums: M = 128, N = n + 1
//              padded to 16, K = n, terms hi Dhi + hi Dlo + lo Dhi;
//   pointwise  o = L_d e (+ local terms), w = n - B e (the other parts of a
//              point by warp shuffles); w replaces psi in TMEM and o goes
//              into the second accumulator;
//   GEMM 2     D2 = o + D w (three terms again);
//   epilogue   D2 + the Nyquist term, re / im paired across lanes, written
//              to the accumulator (z pass), added to it (y pass), or added
//              and weighted (x pass: pout = weight h psi - weightuv v_pair
//              psi, pout_del = v_pair psi, optional <psi|h psi>, <psi|pout>).
// The derivative matrices (hi and lo, K-major, 128-byte swizzled; one set
// when the three spacings are equal, else one per axis) stay in shared
// memory for the kernel's lifetime.  The psi and field values of a tile are
// brought into a shared-memory stage by cp.async (16-byte, coalesced):
// the next tile's psi as soon as the current tile's staging has read it,
// its fields once the pointwise step is done, so the loads overlap the
// GEMMs and the epilogue.
//
// Scheduling: one persistent launch.  An atomic ticket hands out tasks in
// the order [z tiles][y tiles][x tiles] per group of states, so a state's
// accumulator is still in L2 when the next axis pass reads it.  A y (x)
// tile waits, just before its epilogue, until every z (y) tile of its state
// has been published (a release counter per state and pass).  A task only
// waits on tickets handed out before its own, which running CTAs hold, so
// the schedule cannot deadlock.  Every wait is bounded: a timeout latches
// HFB_ERR_CUDA, raises an abort flag the other CTAs see, drains the CTA's
// MMAs and releases TMEM.
#include <limits.h>
#include <math.h>
#include <string.h>
#include <vector>
#include "hfb_ctx.cuh"
#include "hpsi.cuh"
#include "tc_sm100.cuh"

namespace hfb {

namespace {

constexpr int kHtThreads = 256;      // 8 warps: 4 TMEM lane quarters x 2 sets of 8-point chunks
constexpr int kHtLines = 32;         // lines per tile (x 4 parts = 128 rows)
constexpr int kHtTmemCols = 256;     // 2 CTAs per SM
constexpr uint32_t kColAhi = 0, kColAlo = 64, kColD1 = 128, kColD2 = 192;
// n = L_d psi of 8-point chunk jc parks in the columns the plan leaves free
// (48-63, 112-127, 240-255 for n <= 48)
__host__ __device__ constexpr uint32_t ht_ncol(int jc) {
  return (jc < 2 ? 48u : (jc < 4 ? 112u : 240u)) + 8u * (uint32_t)(jc & 1);
}
constexpr long long kHtWaitLimit = 2000000000LL;

template <int N>
struct HtGeo {
  static constexpr int NB = ((N + 1 + 15) / 16) * 16;   // GEMM 1 width: n outputs + alternating sum
  static constexpr int N2 = ((N + 15) / 16) * 16;       // GEMM 2 width
  static constexpr int NKB = (N + 31) / 32;             // 32-float K blocks of a B row
  static constexpr int KS = N / 8;                      // MMA K steps
  static constexpr int NCH = N / 8;                     // 8-point chunks of a line
  static constexpr int CH0 = (NCH + 1) / 2;             // chunks per thread (chunk 2 k + h, h = warp / 4)
  static constexpr int T = N * N / kHtLines;            // tiles per state and axis
  static constexpr uint32_t BTILE = NKB * NB * 128;     // one hi or lo B tile (bytes)
  static constexpr uint32_t BAXIS = 2 * BTILE;
  // shared-memory stage of one tile: psi of both components, the pass's
  // fields and (z pass) the local fields
  static constexpr int PSL = N + 2;                     // z pass: complex per line (16-byte pad)
  static constexpr int PSC_Z = kHtLines * PSL;
  static constexpr int PSC_YX = N * kHtLines;           // y, x passes: [point][line]
  // complex per component, = 8 (mod 16) so the two components' rows of a
  // y / x tile fall into opposite halves of the banks
  static constexpr int PSC = ((PSC_Z > PSC_YX ? PSC_Z : PSC_YX) + 15) / 16 * 16 + 8;
  static constexpr int FL = N + 1;                      // z pass: float4 per line
  static constexpr int FSZ = kHtLines * FL;             // float4 per field buffer (>= 32 n)
  static constexpr size_t STAGE = (size_t)2 * PSC * 8 + (size_t)2 * FSZ * 16;
  static constexpr size_t smem(int nbmat) { return (size_t)nbmat * BAXIS + STAGE + 1024; }
  static_assert(PSC % 2 == 0 && PSL % 2 == 0, "16-byte cp.async destinations");
  static_assert(N % 8 == 0 && (N * N) % kHtLines == 0, "grid size");
  static_assert(NB <= 64 && N2 <= 48 && N <= 64, "TMEM column plan");
  static_assert((NB * 128) % 1024 == 0, "B tile blocks stay 1024-byte aligned");
};

struct HtArgs {
  const float4* F;           // [2][4][n^3] repacked fields (ht_fields_kernel)
  const float* pot;          // [2][12][n^3]
  const float2* psi;
  float2* acc;
  const unsigned char* bmat; // [1 or 3 axes][hi, lo] B tiles
  uint32_t bstride;          // bytes between the axes' B tiles (0: one set for all axes)
  uint32_t bbytes;           // bytes of B tiles to bring in
  int s0, ns, nneut, group;
  float nq[3];               // (pi/d)^2 / n per axis
  const double* weight;
  const double* weightuv;
  float2* pout;
  float2* pout_mf;
  float2* pout_del;
  double* ovl;
  int* cnt;                  // [0] ticket, [1] abort, [2 + 2 s + p] published tiles of pass p
  int* status;
};

// Fields per grid point as float4, one array per use:
//   0 x pass (B, aq_x, wl_y, wl_z)   1 y pass (B, aq_y, wl_x, wl_z)
//   2 z pass (B, aq_z, wl_x, wl_y)   3 local (upot, spot_x, spot_y, spot_z)
// Also zeroes the scheduling counters of the following hpsi_tc_kernel.
__global__ void ht_fields_kernel(const float* __restrict__ pot, float4* __restrict__ F, size_t n3, int* cnt,
                                 int ncnt) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < (size_t)ncnt) cnt[i] = 0;
  if (i >= 2 * n3) return;
  const size_t iq = i / n3, g = i - iq * n3;
  const float* p = pot + iq * 12 * n3;
  const float bm = p[n3 + g], w0 = p[9 * n3 + g], w1 = p[10 * n3 + g], w2 = p[11 * n3 + g];
  float4* f = F + iq * 4 * n3;
  f[g] = make_float4(bm, p[3 * n3 + g], w1, w2);
  f[n3 + g] = make_float4(bm, p[4 * n3 + g], w0, w2);
  f[2 * n3 + g] = make_float4(bm, p[5 * n3 + g], w0, w1);
  f[3 * n3 + g] = make_float4(p[g], p[6 * n3 + g], p[7 * n3 + g], p[8 * n3 + g]);
}

// The lane's part of L_d x (x given by the other parts of the point: u the
// opposite re/im of the own component, v the same re/im and w the opposite
// re/im of the other component).  With L_d x_c = i alpha_c x_c + (beta_c +
// i gamma_c) x_cbar this is sigma alpha_c u + beta_c v + sigma gamma_c w,
// sigma = -1 for a real part, +1 for an imaginary part; kappa = +1 for the
// upper, -1 for the lower component.  sh = sigma/2, kh = kappa/2,
// skh = sigma kappa/2.  Coefficients (h = 1/2), meanfield.py:63-141:
//   z: alpha = -h aq_z,              beta = kappa h wl_x, gamma = -h wl_y
//   y: alpha = -h (aq_y + kappa wl_x), beta = 0,          gamma = h wl_z
//   x: alpha = -h (aq_x - kappa wl_y), beta = -kappa h wl_z, gamma = 0
template <int AX>
__device__ __forceinline__ float ht_lop(float4 f, float sh, float kh, float skh, float u, float v, float w) {
  if (AX == 2) return -sh * f.y * u + kh * f.z * v - sh * f.w * w;
  if (AX == 1) return -(sh * f.y + skh * f.z) * u + sh * f.w * w;
  return -(sh * f.y - skh * f.z) * u - kh * f.w * v;
}

// tf32 rounding (nearest, ties away) on the bit pattern of a finite float
__device__ __forceinline__ float ht_tf32(float x) { return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xffffe000u); }

// D(dcol) (+)= A(TMEM) B^T, three-term tf32 over K = n
template <int N>
__device__ __forceinline__ void ht_gemm(uint32_t tb, uint32_t dcol, uint32_t bhi, int nmma, bool acc0) {
  using G = HtGeo<N>;
  const uint32_t idesc = tc::idesc_tf32(128, nmma);
  const uint32_t blo = bhi + G::BTILE;
#pragma unroll
  for (int ks = 0; ks < G::KS; ++ks) {
    const uint32_t boff = (uint32_t)(ks >> 2) * G::NB * 128 + (uint32_t)(ks & 3) * 32;
    const uint64_t dh = tc::sw128_desc(bhi + boff), dl = tc::sw128_desc(blo + boff);
    tc::mma_tf32_ta(tb + dcol, tb + kColAlo + ks * 8, dh, idesc, (acc0 || ks > 0) ? 1u : 0u);
    tc::mma_tf32_ta(tb + dcol, tb + kColAhi + ks * 8, dl, idesc, 1u);
    tc::mma_tf32_ta(tb + dcol, tb + kColAhi + ks * 8, dh, idesc, 1u);
  }
}

// Wait until *cnt >= target (acquire); false on abort or timeout.
__device__ __forceinline__ bool ht_wait_count(const int* cnt, const int* abort_flag, int target) {
  const long long t0 = clock64();
  for (;;) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(cnt) : "memory");
    if (v >= target) return true;
    if (*(const volatile int*)abort_flag) return false;
    if (clock64() - t0 > kHtWaitLimit) return false;
    __nanosleep(100);
  }
}

struct HtThread {
  int row, ln, c, ri, h, warp;
  uint32_t tb, tl;
  float sh, kh, skh, kp, sk;
};

struct HtShared {
  uint64_t bar_b, bar_mma;
  uint32_t tmem_base;
  int task, next, bad;
  float bsum[2][128];
  double red[8][2];
};

__device__ __forceinline__ void cp16(void* sdst, const void* gsrc) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(tc::smem_u32(sdst)), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Next ticket (INT_MAX once another CTA has aborted).
__device__ __forceinline__ int ht_ticket(const HtArgs& a) {
  int k = atomicAdd(a.cnt, 1);
  if (*(volatile int*)(a.cnt + 1)) k = INT_MAX;
  return k;
}

// Task -> (pass, state, tile); tasks run [z tiles][y tiles][x tiles] per
// group of ``group`` states.  False past the last task.
template <int N>
__device__ __forceinline__ bool ht_decode(const HtArgs& a, int task, int& pass, int& s, int& tile) {
  constexpr int T = HtGeo<N>::T;
  const int gsz = a.group;
  const int nfull = a.ns / gsz;
  const int full_tasks = nfull * 3 * gsz * T;
  if (task >= 3 * a.ns * T) return false;
  int gi, rem, gs;
  if (task < full_tasks) {
    gi = task / (3 * gsz * T);
    rem = task - gi * 3 * gsz * T;
    gs = gsz;
  } else {
    gi = nfull;
    rem = task - full_tasks;
    gs = a.ns - nfull * gsz;
  }
  pass = rem / (gs * T);
  const int r2 = rem - pass * gs * T;
  s = a.s0 + gi * gsz + r2 / T;
  tile = r2 % T;
  return true;
}

// First grid point of line L of a tile along axis AX and the point stride.
template <int N, int AX>
__device__ __forceinline__ size_t ht_line_base(int L) {
  return AX == 2 ? (size_t)L * N : (AX == 1 ? (size_t)(L / N) * N * N + (L % N) : (size_t)L);
}

// psi of both components of a tile -> stage (z: [c][line][point], y / x:
// [c][point][line]); 16-byte copies of 2 consecutive points (z) or lines.
template <int N, int AX>
__device__ __forceinline__ void ht_fetch_psi(const HtArgs& a, float2* ps, int s, int tile) {
  using G = HtGeo<N>;
  constexpr size_t N3 = (size_t)N * N * N;
  constexpr size_t STRIDE = AX == 2 ? 1 : (AX == 1 ? (size_t)N : (size_t)N * N);
  const int L0 = tile * kHtLines;
  for (int e = threadIdx.x; e < 32 * N; e += kHtThreads) {
    const int c = e / (16 * N), r = e - c * 16 * N;
    const float2* src = a.psi + ((size_t)s * 2 + c) * N3;
    float2* dst = ps + c * G::PSC;
    if (AX == 2) {
      const int ln = r / (N / 2), jp = r - ln * (N / 2);
      cp16(dst + ln * G::PSL + 2 * jp, src + (size_t)(L0 + ln) * N + 2 * jp);
    } else {
      const int j = r / 16, lp = r - j * 16;
      cp16(dst + j * kHtLines + 2 * lp, src + ht_line_base<N, AX>(L0 + 2 * lp) + (size_t)j * STRIDE);
    }
  }
}

// The pass's fields (and the local fields for z) of a tile -> stage
// (z: [line][point], y / x: [point][line]).
template <int N, int AX>
__device__ __forceinline__ void ht_fetch_fields(const HtArgs& a, float4* fs, float4* fls, int s, int tile) {
  using G = HtGeo<N>;
  constexpr size_t N3 = (size_t)N * N * N;
  constexpr size_t STRIDE = AX == 2 ? 1 : (AX == 1 ? (size_t)N : (size_t)N * N);
  const int iq = s >= a.nneut ? 1 : 0;
  const float4* F = a.F + ((size_t)iq * 4 + AX) * N3;
  const int L0 = tile * kHtLines;
  for (int e = threadIdx.x; e < kHtLines * N; e += kHtThreads) {
    if (AX == 2) {
      const int ln = e / N, j = e - ln * N;
      const size_t g = (size_t)(L0 + ln) * N + j;
      cp16(fs + ln * G::FL + j, F + g);
      cp16(fls + ln * G::FL + j, F + N3 + g);   // array 3 (local) follows array 2 (z pass)
    } else {
      const int j = e / kHtLines, ln = e - j * kHtLines;
      cp16(fs + j * kHtLines + ln, F + ht_line_base<N, AX>(L0 + ln) + (size_t)j * STRIDE);
    }
  }
}

template <int N>
__device__ __forceinline__ void ht_fetch(const HtArgs& a, int what, float2* ps, float4* fs, float4* fls, int task) {
  int pass, s, tile;
  if (!ht_decode<N>(a, task, pass, s, tile)) return;
  if (what == 0) {
    if (pass == 0) ht_fetch_psi<N, 2>(a, ps, s, tile);
    else if (pass == 1) ht_fetch_psi<N, 1>(a, ps, s, tile);
    else ht_fetch_psi<N, 0>(a, ps, s, tile);
  } else {
    if (pass == 0) ht_fetch_fields<N, 2>(a, fs, fls, s, tile);
    else if (pass == 1) ht_fetch_fields<N, 1>(a, fs, fls, s, tile);
    else ht_fetch_fields<N, 0>(a, fs, fls, s, tile);
  }
}

template <int N, int AX, int P>
__device__ __forceinline__ void ht_tile(const HtArgs& a, const HtThread& t, HtShared& sh, uint32_t bsm, float2* ps,
                                        float4* fs, float4* fls, int s, int tile, int next, uint32_t& phase,
                                        bool& b_ready) {
  using G = HtGeo<N>;
  constexpr size_t N3 = (size_t)N * N * N;
  constexpr size_t STRIDE = AX == 2 ? 1 : (AX == 1 ? (size_t)N : (size_t)N * N);
  const int iq = s >= a.nneut ? 1 : 0;
  const size_t base = ht_line_base<N, AX>(tile * kHtLines + t.ln);
  const uint32_t bhi = bsm + AX * a.bstride;
  // stage indices of point j of the thread's line
  auto pidx = [&](int j) { return AX == 2 ? t.ln * G::PSL + j : j * kHtLines + t.ln; };
  auto fidx = [&](int j) { return AX == 2 ? t.ln * G::FL + j : j * kHtLines + t.ln; };
  const float2* pown = ps + t.c * G::PSC;
  const float2* poth = ps + (1 - t.c) * G::PSC;

  // ---- staging: psi -> TMEM (hi, lo); n = L_d psi -> TMEM; local terms -> D2
#pragma unroll
  for (int k = 0; k < G::CH0; ++k) {
    if (k < G::NCH / 2 || t.h == 0) {
      const int j0 = (2 * k + t.h) * 8;
      float hi[8], lo[8], nv[8], qv[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int j = j0 + i;
        const float2 ov = pown[pidx(j)], tv = poth[pidx(j)];
        const float4 f = fs[fidx(j)];
        const float sv = t.ri ? ov.y : ov.x, u = t.ri ? ov.x : ov.y;
        const float v = t.ri ? tv.y : tv.x, w = t.ri ? tv.x : tv.y;
        nv[i] = ht_lop<AX>(f, t.sh, t.kh, t.skh, u, v, w);
        if (AX == 2) {
          // upot psi + sigma.spot psi (meanfield.py:47-58)
          const float4 g = fls[fidx(j)];
          qv[i] = (g.x + t.kp * g.w) * sv + g.y * v - t.sk * g.z * w;
        }
        hi[i] = ht_tf32(sv);
        lo[i] = sv - hi[i];
      }
      tc::tmem_st8(t.tl + kColAhi + j0, hi);
      tc::tmem_st8(t.tl + kColAlo + j0, lo);
      tc::tmem_st8(t.tl + ht_ncol(2 * k + t.h), nv);
      if (AX == 2) tc::tmem_st8(t.tl + kColD2 + j0, qv);
    }
  }
  tc::tmem_st_wait();
  tc::fence_before();
  __syncthreads();
  // ---- GEMM 1: e = D psi, alternating sums in column n
  if (threadIdx.x == 0) {
    tc::fence_after();
    if (!b_ready) {
      if (!tc::mbar_wait(&sh.bar_b, 0, kHtWaitLimit)) sh.bad = 1;
      b_ready = true;
    }
    ht_gemm<N>(t.tb, kColD1, bhi, G::NB, false);
    tc::mma_commit(&sh.bar_mma);
  }
  // the psi stage is free: bring in the next tile's psi
  ht_fetch<N>(a, 0, ps, fs, fls, next);
  cp_commit();
  // one thread polls the MMA barrier; the others wait at the CTA barrier
  if (threadIdx.x == 0 && !tc::mbar_wait(&sh.bar_mma, phase & 1, kHtWaitLimit)) sh.bad = 1;
  ++phase;
  __syncthreads();
  tc::fence_after();
  // ---- pointwise: o = L_d e (+ local) into D2, w = n - B e into TMEM (A)
  float alt;
  {
    float t8[8];
    tc::tmem_ld8(t.tl + kColD1 + N, t8);
    alt = t8[0];
  }
  float bsum = 0.f;
#pragma unroll
  for (int k = 0; k < G::CH0; ++k) {
    if (k < G::NCH / 2 || t.h == 0) {
      const int j0 = (2 * k + t.h) * 8;
      float e[8], nv[8], hi[8], lo[8], o[8];
      tc::tmem_ld8(t.tl + kColD1 + j0, e);
      tc::tmem_ld8(t.tl + ht_ncol(2 * k + t.h), nv);
      if (AX == 2) tc::tmem_ld8(t.tl + kColD2 + j0, o);
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const float4 f = fs[fidx(j0 + i)];
        const float ue = __shfl_xor_sync(0xffffffffu, e[i], 1);
        const float ve = __shfl_xor_sync(0xffffffffu, e[i], 2);
        const float we = __shfl_xor_sync(0xffffffffu, e[i], 3);
        const float ov = ht_lop<AX>(f, t.sh, t.kh, t.skh, ue, ve, we);
        o[i] = AX == 2 ? o[i] + ov : ov;
        const float wv = nv[i] - f.x * e[i];
        bsum += f.x;
        hi[i] = ht_tf32(wv);
        lo[i] = wv - hi[i];
      }
      tc::tmem_st8(t.tl + kColAhi + j0, hi);
      tc::tmem_st8(t.tl + kColAlo + j0, lo);
      tc::tmem_st8(t.tl + kColD2 + j0, o);
    }
  }
  sh.bsum[t.h][t.row] = bsum;
  tc::tmem_st_wait();
  tc::fence_before();
  __syncthreads();
  // ---- GEMM 2: D2 = o + D w; then wait for the previous pass of this state
  if (threadIdx.x == 0) {
    tc::fence_after();
    ht_gemm<N>(t.tb, kColD2, bhi, G::N2, true);
    tc::mma_commit(&sh.bar_mma);
    if (P > 0 && !ht_wait_count(a.cnt + 2 + 2 * (s - a.s0) + (P - 1), a.cnt + 1, G::T)) {
      sh.bad = 1;
      latch_error(a.status, HFB_ERR_CUDA);
      atomicExch(a.cnt + 1, 1);
    }
  }
  // the field stage is free: bring in the next tile's fields
  ht_fetch<N>(a, 1, ps, fs, fls, next);
  cp_commit();
  if (threadIdx.x == 0 && !tc::mbar_wait(&sh.bar_mma, phase & 1, kHtWaitLimit)) sh.bad = 1;
  ++phase;
  __syncthreads();
  tc::fence_after();
  // ---- epilogue: D2 + Nyquist term, re/im paired across lanes
  const float bbar = (sh.bsum[0][t.row] + sh.bsum[1][t.row]) * (1.f / N);
  const float nyq = a.nq[AX] * bbar * alt;
  const size_t cbase = ((size_t)s * 2 + t.c) * N3 + base;
  float2 zz[G::CH0][4];
#pragma unroll
  for (int k = 0; k < G::CH0; ++k) {
    if (k < G::NCH / 2 || t.h == 0) {
      const int j0 = (2 * k + t.h) * 8;
      float v[8];
      tc::tmem_ld8(t.tl + kColD2 + j0, v);
#pragma unroll
      for (int i = 0; i < 8; ++i) v[i] += (i & 1) ? -nyq : nyq;   // (-1)^j, j0 even
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const float send = t.ri ? v[i] : v[4 + i];
        const float recv = __shfl_xor_sync(0xffffffffu, send, 1);
        zz[k][i] = t.ri ? make_float2(recv, v[4 + i]) : make_float2(v[i], recv);
      }
    }
  }
  // zz[k][i] is the point (2 k + h) * 8 + 4 ri + i of component c
  auto gidx = [&](int k, int i) { return cbase + (size_t)((2 * k + t.h) * 8 + 4 * t.ri + i) * STRIDE; };
  if (P == 0) {
#pragma unroll
    for (int k = 0; k < G::CH0; ++k) {
      if (k < G::NCH / 2 || t.h == 0) {
        float4* d4 = reinterpret_cast<float4*>(a.acc + gidx(k, 0));
        d4[0] = make_float4(zz[k][0].x, zz[k][0].y, zz[k][1].x, zz[k][1].y);
        d4[1] = make_float4(zz[k][2].x, zz[k][2].y, zz[k][3].x, zz[k][3].y);
      }
    }
    // publish this tile for the y pass of the state
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(a.cnt + 2 + 2 * (s - a.s0), 1);
    }
  } else if (P == 1) {
    float2 old[G::CH0][4];
#pragma unroll
    for (int k = 0; k < G::CH0; ++k)
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (k < G::NCH / 2 || t.h == 0) old[k][i] = __ldcg(a.acc + gidx(k, i));
#pragma unroll
    for (int k = 0; k < G::CH0; ++k)
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (k < G::NCH / 2 || t.h == 0) a.acc[gidx(k, i)] = old[k][i] + zz[k][i];
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(a.cnt + 2 + 2 * (s - a.s0) + 1, 1);
    }
  } else {
    // x pass: h psi complete; weights, v_pair psi, overlaps
    const float wt = a.weight ? (float)a.weight[s] : 1.f;
    const float wu = a.weightuv ? (float)a.weightuv[s] : 0.f;
    const float* vpq = a.pot + ((size_t)iq * 12 + 2) * N3 + base;
    const float2* own = a.psi + cbase;
    float2 old[G::CH0][4], psv[G::CH0][4];
    float vpv[G::CH0][4];
#pragma unroll
    for (int k = 0; k < G::CH0; ++k)
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (k < G::NCH / 2 || t.h == 0) {
          const size_t o = (size_t)((2 * k + t.h) * 8 + 4 * t.ri + i) * STRIDE;
          old[k][i] = __ldcg(a.acc + cbase + o);
          psv[k][i] = __ldg(own + o);
          vpv[k][i] = __ldg(vpq + o);
        }
    double ov_mf = 0.0, ov_po = 0.0;
#pragma unroll
    for (int k = 0; k < G::CH0; ++k)
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (k < G::NCH / 2 || t.h == 0) {
          const size_t gi = gidx(k, i);
          const float2 mf = old[k][i] + zz[k][i];
          const float2 ps_ = psv[k][i];
          const float2 dl = vpv[k][i] * ps_;
          const float2 po = wt * mf - wu * dl;
          if (a.pout_mf) a.pout_mf[gi] = mf;
          if (a.pout) a.pout[gi] = po;
          if (a.pout_del) a.pout_del[gi] = dl;
          ov_mf += (double)ps_.x * (double)mf.x + (double)ps_.y * (double)mf.y;
          ov_po += (double)ps_.x * (double)po.x + (double)ps_.y * (double)po.y;
        }
    if (a.ovl) {
      // deterministic per-tile partial sums: warp shuffles, then thread 0
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        ov_mf += __shfl_xor_sync(0xffffffffu, ov_mf, o);
        ov_po += __shfl_xor_sync(0xffffffffu, ov_po, o);
      }
      if ((threadIdx.x & 31) == 0) {
        sh.red[t.warp][0] = ov_mf;
        sh.red[t.warp][1] = ov_po;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        double x = 0.0, y = 0.0;
        for (int w = 0; w < kHtThreads / 32; ++w) {
          x += sh.red[w][0];
          y += sh.red[w][1];
        }
        a.ovl[((size_t)(s - a.s0) * G::T + tile) * 2 + 0] = x;
        a.ovl[((size_t)(s - a.s0) * G::T + tile) * 2 + 1] = y;
      }
    }
  }
}

template <int N>
__global__ void __launch_bounds__(kHtThreads, 2) hpsi_tc_kernel(HtArgs a) {
  using G = HtGeo<N>;
  extern __shared__ unsigned char ht_smem_raw[];
  __shared__ HtShared sh;
  unsigned char* bs = reinterpret_cast<unsigned char*>(((uintptr_t)ht_smem_raw + 1023) & ~(uintptr_t)1023);
  float2* ps = reinterpret_cast<float2*>(bs + a.bbytes);
  float4* fs = reinterpret_cast<float4*>(ps + 2 * G::PSC);
  float4* fls = fs + G::FSZ;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) {
    tc::tmem_alloc(&sh.tmem_base, kHtTmemCols);
    tc::tmem_relinquish();
  }
  if (tid == 0) {
    sh.bad = 0;
    tc::mbar_init(&sh.bar_b, 1);
    tc::mbar_init(&sh.bar_mma, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    tc::mbar_arrive_expect_tx(&sh.bar_b, a.bbytes);
    tc::bulk_g2s(bs, a.bmat, a.bbytes, &sh.bar_b);
    sh.task = ht_ticket(a);
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();

  HtThread t;
  t.warp = warp;
  const int q = warp & 3;
  t.h = warp >> 2;
  t.row = 32 * q + lane;
  t.ln = t.row >> 2;
  t.c = (t.row >> 1) & 1;
  t.ri = t.row & 1;
  t.tb = sh.tmem_base;
  t.tl = t.tb + ((uint32_t)(32 * q) << 16);
  const float sg = t.ri ? 1.f : -1.f;
  t.kp = t.c ? -1.f : 1.f;
  t.sh = 0.5f * sg;
  t.kh = 0.5f * t.kp;
  t.skh = 0.5f * sg * t.kp;
  t.sk = sg * t.kp;
  const uint32_t bsm = tc::smem_u32(bs);

  int task = sh.task;
  ht_fetch<N>(a, 0, ps, fs, fls, task);
  ht_fetch<N>(a, 1, ps, fs, fls, task);
  cp_commit();
  uint32_t phase = 0;
  bool b_ready = false;
  for (;;) {
    int pass, s, tile;
    if (!ht_decode<N>(a, task, pass, s, tile)) break;
    if (tid == 0) sh.next = ht_ticket(a);
    cp_wait_all();
    __syncthreads();   // the tile's stage has landed; sh.next is visible
    if (sh.bad) break;
    const int next = sh.next;
    if (pass == 0)
      ht_tile<N, 2, 0>(a, t, sh, bsm, ps, fs, fls, s, tile, next, phase, b_ready);
    else if (pass == 1)
      ht_tile<N, 1, 1>(a, t, sh, bsm, ps, fs, fls, s, tile, next, phase, b_ready);
    else
      ht_tile<N, 0, 2>(a, t, sh, bsm, ps, fs, fls, s, tile, next, phase, b_ready);
    task = next;
  }
  cp_wait_all();   // no copy may land after the CTA has gone
  tc::fence_before();
  __syncthreads();
  if (sh.bad) {
    if (tid == 0) {
      latch_error(a.status, HFB_ERR_CUDA);
      atomicExch(a.cnt + 1, 1);
      if (phase > 0) tc::mbar_wait(&sh.bar_mma, (phase - 1) & 1, kHtWaitLimit);
      if (!b_ready) tc::mbar_wait(&sh.bar_b, 0, kHtWaitLimit);
    }
    __syncthreads();
  } else if (tid == 0 && !b_ready) {
    // no task ran: let the B copy land before the CTA exits
    tc::mbar_wait(&sh.bar_b, 0, kHtWaitLimit);
  }
  if (warp == 0) {
    tc::fence_after();
    tc::tmem_dealloc(t.tb, kHtTmemCols);
  }
}

float tf32_host(float x) {
  uint32_t u;
  memcpy(&u, &x, 4);
  if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & 0xffffe000u;
  float r;
  memcpy(&r, &u, 4);
  return r;
}

uint32_t sw128_host(int r, int c) { return (uint32_t)((r >> 3) * 1024 + (r & 7) * 128 + ((c ^ (r & 7)) << 4)); }

// B tiles of the three axes: row m < n holds D[m][:] (the spectral first
// derivative with the k = 0 and n/2 bins zeroed, -(2 kf / n) sum_{k=1}^{n/2-1}
// k sin(2 pi k (m - l) / n), kf = 2 pi / (n d)), row n the alternating signs,
// further rows zero; hi = tf32(D), lo = tf32(D - hi).
template <int N>
int hpsi_tc_prepare_t(hfb_ctx_s* c) {
  using G = HtGeo<N>;
  constexpr uint32_t BALL = 3 * G::BAXIS;
  std::vector<unsigned char> img(BALL, 0);
  for (int ax = 0; ax < 3; ++ax) {
    const double kf = 2.0 * kPi / (N * c->d[ax]);
    for (int row = 0; row < G::NB; ++row)
      for (int l = 0; l < N; ++l) {
        double v = 0.0;
        if (row < N) {
          for (int k = 1; k < N / 2; ++k) {
            const int ph = (((k * (row - l)) % N) + N) % N;
            v += k * sin(2.0 * kPi * ph / N);
          }
          v *= -2.0 * kf / N;
        } else if (row == N) {
          v = (l & 1) ? -1.0 : 1.0;
        }
        const float hi = tf32_host((float)v);
        const float lo = tf32_host((float)(v - (double)hi));
        const size_t off = (size_t)(l / 32) * G::NB * 128 + sw128_host(row, (l % 32) / 4) + (l % 4) * 4;
        memcpy(&img[ax * G::BAXIS + off], &hi, 4);
        memcpy(&img[ax * G::BAXIS + G::BTILE + off], &lo, 4);
      }
  }
  if (cudaMalloc(&c->hpsi_b, BALL) != cudaSuccess) {
    cudaGetLastError();
    c->hpsi_b = nullptr;
    return HFB_ERR_ALLOC;
  }
  if (cudaMemcpy(c->hpsi_b, img.data(), BALL, cudaMemcpyHostToDevice) != cudaSuccess) return HFB_ERR_CUDA;
  return HFB_OK;
}

int sm_count() {
  static const int n = [] {
    int d = 0, v = 0;
    cudaGetDevice(&d);
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, d);
    return v > 0 ? v : 1;
  }();
  return n;
}

template <int N>
int hpsi_tc_launch_t(hfb_ctx_s* c, const void* pot, int s0, int ns, int nneut, const void* psi,
                     const double* weight, const double* weightuv, void* acc, void* pout, void* pout_mf,
                     void* pout_del, double* ovl, cudaStream_t st) {
  using G = HtGeo<N>;
  constexpr size_t N3 = (size_t)N * N * N;
  const size_t fbytes = sizeof(float4) * 8 * N3;
  const int ncnt = 2 + 2 * ns;
  unsigned char* scr = (unsigned char*)scratch(c, hfb_ctx_s::S_HPT, fbytes + sizeof(int) * (size_t)ncnt);
  if (!scr) return HFB_ERR_ALLOC;
  float4* F = reinterpret_cast<float4*>(scr);
  int* cnt = reinterpret_cast<int*>(scr + fbytes);
  const size_t tot = 2 * N3 > (size_t)ncnt ? 2 * N3 : (size_t)ncnt;
  ht_fields_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>((const float*)pot, F, N3, cnt, ncnt);
  HFB_CHECK_LAUNCH();
  const int slots = 2 * sm_count();
  int group = (slots + G::T / 2) / G::T;
  if (group < 1) group = 1;
  if (group > ns) group = ns;
  const int ntask = 3 * ns * G::T;
  HtArgs a;
  a.F = F;
  a.pot = (const float*)pot;
  a.psi = (const float2*)psi;
  a.acc = (float2*)acc;
  a.bmat = c->hpsi_b;
  const bool uniform = c->d[0] == c->d[1] && c->d[1] == c->d[2];
  a.bstride = uniform ? 0u : G::BAXIS;
  a.bbytes = uniform ? G::BAXIS : 3u * G::BAXIS;
  a.s0 = s0;
  a.ns = ns;
  a.nneut = nneut;
  a.group = group;
  for (int ax = 0; ax < 3; ++ax) a.nq[ax] = (float)((kPi / c->d[ax]) * (kPi / c->d[ax]) / N);
  a.weight = weight;
  a.weightuv = weightuv;
  a.pout = (float2*)pout;
  a.pout_mf = (float2*)pout_mf;
  a.pout_del = (float2*)pout_del;
  a.ovl = ovl;
  a.cnt = cnt;
  a.status = c->dev_status;
  allow_max_dynamic_smem(hpsi_tc_kernel<N>);
  hpsi_tc_kernel<N><<<ntask < slots ? ntask : slots, kHtThreads, G::smem(uniform ? 1 : 3), st>>>(a);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

}  // namespace

int hpsi_tc_prepare(hfb_ctx_s* c) {
  c->hpsi_b = nullptr;
  switch (c->n) {
    case 24: return hpsi_tc_prepare_t<24>(c);
    case 32: return hpsi_tc_prepare_t<32>(c);
    case 40: return hpsi_tc_prepare_t<40>(c);
    case 48: return hpsi_tc_prepare_t<48>(c);
    default: return HFB_OK;   // other grids keep the FFT path
  }
}

bool hpsi_tc_available(hfb_ctx_s* c, int prec) { return prec == HFB_F32 && c->use_tcgen05 && c->hpsi_b; }

int hpsi_tc_parts(hfb_ctx_s* c) { return c->n * c->n / kHtLines; }

int hpsi_tc_launch(hfb_ctx_s* c, const void* pot, int s0, int ns, int nneut, const void* psi, const double* weight,
                   const double* weightuv, void* acc, void* pout, void* pout_mf, void* pout_del, double* ovl,
                   cudaStream_t st) {
  if (ns <= 0) return HFB_OK;
  switch (c->n) {
    case 24: return hpsi_tc_launch_t<24>(c, pot, s0, ns, nneut, psi, weight, weightuv, acc, pout, pout_mf, pout_del, ovl, st);
    case 32: return hpsi_tc_launch_t<32>(c, pot, s0, ns, nneut, psi, weight, weightuv, acc, pout, pout_mf, pout_del, ovl, st);
    case 40: return hpsi_tc_launch_t<40>(c, pot, s0, ns, nneut, psi, weight, weightuv, acc, pout, pout_mf, pout_del, ovl, st);
    case 48: return hpsi_tc_launch_t<48>(c, pot, s0, ns, nneut, psi, weight, weightuv, acc, pout, pout_mf, pout_del, ovl, st);
    default: return HFB_ERR_UNSUPPORTED_GRID;
  }
}

}  // namespace hfb
