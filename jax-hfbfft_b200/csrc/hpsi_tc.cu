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
// The Nyquist term is (pi/d)^2 mean_line(B) (-1)^j sum_l (-1)^l psi_l / n.
//
// A tile is 64 lines of one axis of one state: 128 GEMM rows, row = 2 line
// + spinor component, so a thread owns whole complex values of one
// component and finds the other component in the neighbouring lane.  Real
// and imaginary parts sit in separate TMEM column blocks and are two GEMMs
// against the same B.
//   staging    each thread (row, every fourth 4-point chunk) reads psi from
//              the shared-memory stage, computes n = L_d psi and its part of
//              the alternating sums and of the mean of B (parked in spare
//              TMEM columns), for the z pass the local upot / spin terms
//              (stored into the second accumulator), splits psi = hi + lo
//              (tf32) and stores both into TMEM, where tcgen05.mma reads its
//              A operand;
//   GEMM 1     e = D psi: M = 128, N = n padded to 16, K = n, for Re and Im,
//              terms hi Dhi + hi Dlo + lo Dhi;
//   pointwise  o = L_d e (+ local terms), w = n - B e; w replaces psi in
//              TMEM and o goes into the second accumulator;
//   GEMM 2     D2 = o + D w;
//   epilogue   D2 + the Nyquist term, written to the accumulator (z pass),
//              added to it (y pass), or added and weighted (x pass: pout =
//              weight h psi - weightuv v_pair psi, pout_del = v_pair psi,
//              optional <psi|h psi>, <psi|pout>).
// The derivative matrices (hi and lo, K-major, 128-byte swizzled; one set
// when the three spacings are equal, else one per axis) stay in shared
// memory for the kernel's lifetime.  The psi and field values of a tile are
// brought into the stage by cp.async (coalesced): the next tile's psi as
// soon as the current tile's staging has read it, its fields once the
// pointwise step is done, so the loads overlap the GEMMs and the epilogue.
//
// Scheduling: one persistent launch, one 512-thread CTA per SM (all 512
// TMEM columns).  An atomic ticket hands out tasks in the order [z tiles]
// [y tiles][x tiles] per group of states, so a state's accumulator is still
// in L2 when the next axis pass reads it.  A y (x) tile waits, just before
// its epilogue, until every z (y) tile of its state has been published (a
// release counter per state and pass).  A task only waits on tickets handed
// out before its own, which running CTAs hold (as current or prefetched
// task), so the schedule cannot deadlock.  Every wait is bounded: a timeout
// latches HFB_ERR_CUDA, raises an abort flag the other CTAs see, drains the
// CTA's MMAs and copies and releases TMEM.
#include <limits.h>
#include <math.h>
#include <string.h>
#include <vector>
#include "hfb_ctx.cuh"
#include "hpsi.cuh"
#include "tc_sm100.cuh"

namespace hfb {

namespace {

constexpr int kHtThreads = 512;      // 16 warps: 4 TMEM lane quarters x 4 groups of chunks
constexpr int kHtWarps = kHtThreads / 32;
constexpr int kHtLines = 64;         // lines per tile (x 2 components = 128 rows)
constexpr int kHtTmemCols = 512;
// TMEM, 64-column slots: psi / w (hi re, hi im, lo re, lo im), D1 = D psi
// (re, im), D2 = o + D w (re, im)
constexpr uint32_t kAHR = 0, kAHI = 64, kALR = 128, kALI = 192, kD1R = 256, kD1I = 320, kD2R = 384, kD2I = 448;
// n = L_d psi of 4-point chunk jc parks in columns 48-63 of slots 0-2 (re)
// and 3-5 (im), which the plan leaves free for n <= 48; columns 432-447
// hold each chunk group's partial alternating sums and sum of B
constexpr uint32_t kRed = 432;
__host__ __device__ constexpr uint32_t ht_ncol(int part, int jc) {
  return 64u * (uint32_t)(3 * part + jc / 4) + 48u + 4u * (uint32_t)(jc % 4);
}
constexpr long long kHtWaitLimit = 2000000000LL;

template <int N>
struct HtGeo {
  static constexpr int N2 = ((N + 15) / 16) * 16;       // MMA width = B rows
  static constexpr int NKB = (N + 31) / 32;             // 32-float K blocks of a B row
  static constexpr int KS = N / 8;                      // MMA K steps
  static constexpr int NCH = N / 4;                     // 4-point chunks of a line
  static constexpr int CHK = (NCH + 3) / 4;             // chunks per thread (chunk 4 k + group)
  static constexpr int T = N * N / kHtLines;            // tiles per state and axis
  static constexpr uint32_t BTILE = NKB * N2 * 128;     // one hi or lo B tile (bytes)
  static constexpr uint32_t BAXIS = 2 * BTILE;
  // stage of one tile
  static constexpr int PRZ = N + 1;                     // z pass: complex per (line, component) row
  static constexpr int PSZ_Z = kHtLines * 2 * PRZ;
  static constexpr int PSC_YX = ((N * kHtLines + 15) / 16) * 16 + 8;  // y, x: per component, [point][line]
  static constexpr int PSZ = PSZ_Z > 2 * PSC_YX ? PSZ_Z : 2 * PSC_YX; // complex
  static constexpr int FL = N + 1;                      // z pass: float4 per line
  static constexpr int FSZ = kHtLines * FL;             // float4 per field buffer (>= 64 n)
  static constexpr size_t STAGE = (size_t)PSZ * 8 + (size_t)2 * FSZ * 16;
  static constexpr size_t smem(int nbmat) { return (size_t)nbmat * BAXIS + STAGE + 1024; }
  static_assert(N % 8 == 0 && (N * N) % kHtLines == 0 && N <= 48, "grid size");
  static_assert((N2 * 128) % 1024 == 0, "B tile blocks stay 1024-byte aligned");
  static_assert(PSZ % 2 == 0, "16-byte aligned field stage");
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

// Fields per grid point as float4, one array per use (current and
// spin-orbit fields halved, as they enter L_d):
//   0 x pass (B, aq_x/2, wl_y/2, wl_z/2)   1 y pass (B, aq_y/2, wl_x/2, wl_z/2)
//   2 z pass (B, aq_z/2, wl_x/2, wl_y/2)   3 local (upot, spot_x, spot_y, spot_z)
// Also zeroes the scheduling counters of the following hpsi_tc_kernel.
__global__ void ht_fields_kernel(const float* __restrict__ pot, float4* __restrict__ F, size_t n3, int* cnt,
                                 int ncnt) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < (size_t)ncnt) cnt[i] = 0;
  if (i >= 2 * n3) return;
  const size_t iq = i / n3, g = i - iq * n3;
  const float* p = pot + iq * 12 * n3;
  const float bm = p[n3 + g];
  const float w0 = 0.5f * p[9 * n3 + g], w1 = 0.5f * p[10 * n3 + g], w2 = 0.5f * p[11 * n3 + g];
  float4* f = F + iq * 4 * n3;
  f[g] = make_float4(bm, 0.5f * p[3 * n3 + g], w1, w2);
  f[n3 + g] = make_float4(bm, 0.5f * p[4 * n3 + g], w0, w2);
  f[2 * n3 + g] = make_float4(bm, 0.5f * p[5 * n3 + g], w0, w1);
  f[3 * n3 + g] = make_float4(p[g], p[6 * n3 + g], p[7 * n3 + g], p[8 * n3 + g]);
}

// L_d of the own component: L_d x_c = i alpha_c x_c + (beta_c + i gamma_c)
// x_cbar with (kp = +1 upper, -1 lower component; f the pass's halved
// fields), meanfield.py:63-141:
//   z: alpha = -aq_z/2,               beta = kp wl_x/2,  gamma = -wl_y/2
//   y: alpha = -(aq_y + kp wl_x)/2,   beta = 0,          gamma = wl_z/2
//   x: alpha = -(aq_x - kp wl_y)/2,   beta = -kp wl_z/2, gamma = 0
template <int AX>
__device__ __forceinline__ float2 ht_l(float4 f, float kp, float2 a, float2 b) {
  float2 r;
  if (AX == 2) {
    const float be = kp * f.z;
    r.x = f.y * a.y + be * b.x + f.w * b.y;
    r.y = -f.y * a.x + be * b.y - f.w * b.x;
  } else if (AX == 1) {
    const float al = f.y + kp * f.z;   // -alpha
    r.x = al * a.y - f.w * b.y;
    r.y = -al * a.x + f.w * b.x;
  } else {
    const float al = f.y - kp * f.z;   // -alpha
    const float be = kp * f.w;         // -beta
    r.x = al * a.y - be * b.x;
    r.y = -al * a.x - be * b.y;
  }
  return r;
}

// tf32 rounding (nearest, ties away) on the bit pattern of a finite float
__device__ __forceinline__ float ht_tf32(float x) { return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xffffe000u); }

__device__ __forceinline__ void tmem_ld4(uint32_t taddr, float (&v)[4]) {
  uint32_t r[4];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 4; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_st4(uint32_t taddr, const float (&v)[4]) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1,%2,%3,%4};" ::"r"(taddr),
               "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
               "r"(__float_as_uint(v[3]))
               : "memory");
}

// (D re, D im) (+)= A(TMEM re, im) B^T, three-term tf32 over K = n
template <int N>
__device__ __forceinline__ void ht_gemm(uint32_t tb, uint32_t dre, uint32_t dim, uint32_t bhi, bool acc0) {
  using G = HtGeo<N>;
  const uint32_t idesc = tc::idesc_tf32(128, G::N2);
  const uint32_t blo = bhi + G::BTILE;
#pragma unroll
  for (int ks = 0; ks < G::KS; ++ks) {
    const uint32_t boff = (uint32_t)(ks >> 2) * G::N2 * 128 + (uint32_t)(ks & 3) * 32;
    const uint64_t dh = tc::sw128_desc(bhi + boff), dl = tc::sw128_desc(blo + boff);
    const uint32_t acc = (acc0 || ks > 0) ? 1u : 0u;
    tc::mma_tf32_ta(tb + dre, tb + kALR + ks * 8, dh, idesc, acc);
    tc::mma_tf32_ta(tb + dim, tb + kALI + ks * 8, dh, idesc, acc);
    tc::mma_tf32_ta(tb + dre, tb + kAHR + ks * 8, dl, idesc, 1u);
    tc::mma_tf32_ta(tb + dim, tb + kAHI + ks * 8, dl, idesc, 1u);
    tc::mma_tf32_ta(tb + dre, tb + kAHR + ks * 8, dh, idesc, 1u);
    tc::mma_tf32_ta(tb + dim, tb + kAHI + ks * 8, dh, idesc, 1u);
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
  int row, ln, c, g, warp;
  uint32_t tb, tl;
  float kp;
};

struct HtShared {
  uint64_t bar_b, bar_mma;
  uint32_t tmem_base;
  int task, next, bad;
  double ovr[kHtWarps][2];
};

__device__ __forceinline__ void cp16(void* sdst, const void* gsrc) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(tc::smem_u32(sdst)), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp8(void* sdst, const void* gsrc) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(tc::smem_u32(sdst)), "l"(gsrc) : "memory");
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

// First grid point of line L of a tile along axis AX (points follow at
// stride 1, n, n^2 for AX = 2, 1, 0).
template <int N, int AX>
__device__ __forceinline__ size_t ht_line_base(int L) {
  return AX == 2 ? (size_t)L * N : (AX == 1 ? (size_t)(L / N) * N * N + (L % N) : (size_t)L);
}

// psi of a tile -> stage.  z: [line][component][point] rows of n + 1
// complex, thread -> (row, points j = tid % 4 + 4 m) with 8-byte copies;
// y, x: [component][point][line], thread -> (component, line pair,
// points j = tid / 64 + 8 m) with 16-byte copies of 2 lines.
template <int N, int AX>
__device__ __forceinline__ void ht_fetch_psi(const HtArgs& a, float2* ps, int s, int tile) {
  using G = HtGeo<N>;
  constexpr size_t N3 = (size_t)N * N * N;
  constexpr size_t STRIDE = AX == 2 ? 1 : (AX == 1 ? (size_t)N : (size_t)N * N);
  static_assert(kHtThreads == 4 * 2 * kHtLines && N % 8 == 0, "fetch mapping");
  const int L0 = tile * kHtLines;
  const float2* src = a.psi + (size_t)s * 2 * N3;
  if (AX == 2) {
    const int r = threadIdx.x >> 2, j = threadIdx.x & 3, ln = r >> 1, c = r & 1;
    const float2* g = src + c * N3 + (size_t)(L0 + ln) * N + j;
    float2* d = ps + r * G::PRZ + j;
#pragma unroll
    for (int m = 0; m < N / 4; ++m) cp8(d + 4 * m, g + 4 * m);
  } else {
    const int lp = threadIdx.x & 31, c = (threadIdx.x >> 5) & 1, j = threadIdx.x >> 6;
    const float2* g = src + c * N3 + ht_line_base<N, AX>(L0 + 2 * lp) + (size_t)j * STRIDE;
    float2* d = ps + c * G::PSC_YX + j * kHtLines + 2 * lp;
#pragma unroll
    for (int m = 0; m < N / 8; ++m) cp16(d + 8 * m * kHtLines, g + 8 * m * STRIDE);
  }
}

// The pass's fields (and the local fields for z) of a tile -> stage.
// z: [line][point], thread -> (line, points j = tid % 8 + 8 m); y, x:
// [point][line], thread -> (line, points j = tid / 64 + 8 m).
template <int N, int AX>
__device__ __forceinline__ void ht_fetch_fields(const HtArgs& a, float4* fs, float4* fls, int s, int tile) {
  using G = HtGeo<N>;
  constexpr size_t N3 = (size_t)N * N * N;
  constexpr size_t STRIDE = AX == 2 ? 1 : (AX == 1 ? (size_t)N : (size_t)N * N);
  const int iq = s >= a.nneut ? 1 : 0;
  const float4* F = a.F + ((size_t)iq * 4 + AX) * N3;
  const int L0 = tile * kHtLines;
  if (AX == 2) {
    const int ln = threadIdx.x >> 3, j = threadIdx.x & 7;
    const float4* g = F + (size_t)(L0 + ln) * N + j;
    float4* d = fs + ln * G::FL + j;
    float4* dl = fls + ln * G::FL + j;
#pragma unroll
    for (int m = 0; m < N / 8; ++m) {
      cp16(d + 8 * m, g + 8 * m);
      cp16(dl + 8 * m, g + N3 + 8 * m);   // array 3 (local) follows array 2 (z pass)
    }
  } else {
    const int ln = threadIdx.x & 63, j = threadIdx.x >> 6;
    const float4* g = F + ht_line_base<N, AX>(L0 + ln) + (size_t)j * STRIDE;
    float4* d = fs + j * kHtLines + ln;
#pragma unroll
    for (int m = 0; m < N / 8; ++m) cp16(d + 8 * m * kHtLines, g + 8 * m * STRIDE);
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
  constexpr int PSTEP = AX == 2 ? 1 : kHtLines;   // stage step between consecutive points
  const int iq = s >= a.nneut ? 1 : 0;
  const size_t base = ht_line_base<N, AX>(tile * kHtLines + t.ln);
  const uint32_t bhi = bsm + AX * a.bstride;
  const float2* pa = AX == 2 ? ps + (2 * t.ln + t.c) * G::PRZ : ps + t.c * G::PSC_YX + t.ln;
  const float2* pb = AX == 2 ? ps + (2 * t.ln + 1 - t.c) * G::PRZ : ps + (1 - t.c) * G::PSC_YX + t.ln;
  const float4* fa = AX == 2 ? fs + t.ln * G::FL : fs + t.ln;
  const float4* fl = fls + t.ln * G::FL;

  // ---- staging: psi -> TMEM (hi, lo); n = L_d psi -> TMEM; local terms -> D2
  {
    float4 red = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int k = 0; k < G::CHK; ++k) {
      if (k < G::NCH / 4 || 4 * k + t.g < G::NCH) {
        const int jc = 4 * k + t.g, j0 = 4 * jc;
        float hr[4], hm[4], lr[4], lm[4], nr[4], nm[4], qr[4], qm[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int j = j0 + i;
          const float2 av = pa[j * PSTEP], bv = pb[j * PSTEP];
          const float4 f = fa[j * PSTEP];
          const float2 n = ht_l<AX>(f, t.kp, av, bv);
          nr[i] = n.x;
          nm[i] = n.y;
          if (AX == 2) {
            // upot psi + sigma.spot psi (meanfield.py:47-58)
            const float4 g = fl[j];
            const float d = g.x + t.kp * g.w, s1 = t.kp * g.z;
            qr[i] = d * av.x + g.y * bv.x + s1 * bv.y;
            qm[i] = d * av.y + g.y * bv.y - s1 * bv.x;
          }
          hr[i] = ht_tf32(av.x);
          lr[i] = av.x - hr[i];
          hm[i] = ht_tf32(av.y);
          lm[i] = av.y - hm[i];
          red.x += (i & 1) ? -av.x : av.x;   // (-1)^j psi, j0 even
          red.y += (i & 1) ? -av.y : av.y;
          red.z += f.x;
        }
        tmem_st4(t.tl + kAHR + j0, hr);
        tmem_st4(t.tl + kAHI + j0, hm);
        tmem_st4(t.tl + kALR + j0, lr);
        tmem_st4(t.tl + kALI + j0, lm);
        tmem_st4(t.tl + ht_ncol(0, jc), nr);
        tmem_st4(t.tl + ht_ncol(1, jc), nm);
        if (AX == 2) {
          tmem_st4(t.tl + kD2R + j0, qr);
          tmem_st4(t.tl + kD2I + j0, qm);
        }
      }
    }
    const float rv[4] = {red.x, red.y, red.z, 0.f};
    tmem_st4(t.tl + kRed + 4 * t.g, rv);
  }
  tc::tmem_st_wait();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  // ---- GEMM 1: e = D psi
  if (threadIdx.x == 0) {
    tc::fence_after();
    if (!b_ready) {
      // on a timeout b_ready stays false: the exit path waits for the copy
      if (tc::mbar_wait(&sh.bar_b, 0, kHtWaitLimit)) b_ready = true;
      else sh.bad = 1;
    }
    ht_gemm<N>(t.tb, kD1R, kD1I, bhi, false);
    tc::mma_commit(&sh.bar_mma);
  }
  // the psi stage is free: bring in the next tile's psi
  ht_fetch<N>(a, 0, ps, fs, fls, next);
  cp_commit();
  float2 alt;
  float bbar;
  {
    float r[16];
    tc::tmem_ld16(t.tl + kRed, r);
    alt = make_float2(r[0] + r[4] + r[8] + r[12], r[1] + r[5] + r[9] + r[13]);
    bbar = (r[2] + r[6] + r[10] + r[14]) * (1.f / N);
  }
  // one thread polls the MMA barrier; the others wait at the CTA barrier
  if (threadIdx.x == 0 && !tc::mbar_wait(&sh.bar_mma, phase & 1, kHtWaitLimit)) sh.bad = 1;
  ++phase;
  __syncthreads();
  tc::fence_after();
  // ---- pointwise: o = L_d e (+ local) into D2, w = n - B e into TMEM (A)
#pragma unroll
  for (int k = 0; k < G::CHK; ++k) {
    if (k < G::NCH / 4 || 4 * k + t.g < G::NCH) {
      const int jc = 4 * k + t.g, j0 = 4 * jc;
      float er[4], em[4], nr[4], nm[4], orr[4], om[4], hr[4], hm[4], lr[4], lm[4];
      tmem_ld4(t.tl + kD1R + j0, er);
      tmem_ld4(t.tl + kD1I + j0, em);
      tmem_ld4(t.tl + ht_ncol(0, jc), nr);
      tmem_ld4(t.tl + ht_ncol(1, jc), nm);
      if (AX == 2) {
        tmem_ld4(t.tl + kD2R + j0, orr);
        tmem_ld4(t.tl + kD2I + j0, om);
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const float4 f = fa[(j0 + i) * PSTEP];
        const float2 ev = make_float2(er[i], em[i]);
        const float2 eo = make_float2(__shfl_xor_sync(0xffffffffu, er[i], 1), __shfl_xor_sync(0xffffffffu, em[i], 1));
        const float2 o = ht_l<AX>(f, t.kp, ev, eo);
        orr[i] = AX == 2 ? orr[i] + o.x : o.x;
        om[i] = AX == 2 ? om[i] + o.y : o.y;
        const float wr = nr[i] - f.x * ev.x, wm = nm[i] - f.x * ev.y;
        hr[i] = ht_tf32(wr);
        lr[i] = wr - hr[i];
        hm[i] = ht_tf32(wm);
        lm[i] = wm - hm[i];
      }
      tmem_st4(t.tl + kAHR + j0, hr);
      tmem_st4(t.tl + kAHI + j0, hm);
      tmem_st4(t.tl + kALR + j0, lr);
      tmem_st4(t.tl + kALI + j0, lm);
      tmem_st4(t.tl + kD2R + j0, orr);
      tmem_st4(t.tl + kD2I + j0, om);
    }
  }
  tc::tmem_st_wait();
  tc::fence_before();
  __syncthreads();
  // ---- GEMM 2: D2 = o + D w; then wait for the previous pass of this state
  if (threadIdx.x == 0) {
    tc::fence_after();
    ht_gemm<N>(t.tb, kD2R, kD2I, bhi, true);
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
  // ---- epilogue: D2 + Nyquist term
  const float nyq = a.nq[AX] * bbar;
  const size_t cbase = ((size_t)s * 2 + t.c) * N3 + base;
  float2 zz[G::CHK][4];
#pragma unroll
  for (int k = 0; k < G::CHK; ++k) {
    if (k < G::NCH / 4 || 4 * k + t.g < G::NCH) {
      const int j0 = 4 * (4 * k + t.g);
      float vr[4], vm[4];
      tmem_ld4(t.tl + kD2R + j0, vr);
      tmem_ld4(t.tl + kD2I + j0, vm);
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const float sgn = (i & 1) ? -nyq : nyq;   // (-1)^j, j0 even
        zz[k][i] = make_float2(vr[i] + sgn * alt.x, vm[i] + sgn * alt.y);
      }
    }
  }
  // zz[k][i] is the point 4 (4 k + g) + i of component c
  auto off = [&](int k, int i) { return (size_t)(4 * (4 * k + t.g) + i) * STRIDE; };
  if (P == 0) {
#pragma unroll
    for (int k = 0; k < G::CHK; ++k) {
      if (k < G::NCH / 4 || 4 * k + t.g < G::NCH) {
        float4* d4 = reinterpret_cast<float4*>(a.acc + cbase + off(k, 0));
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
    float2 old[G::CHK][4];
#pragma unroll
    for (int k = 0; k < G::CHK; ++k)
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (k < G::NCH / 4 || 4 * k + t.g < G::NCH) old[k][i] = __ldcg(a.acc + cbase + off(k, i));
#pragma unroll
    for (int k = 0; k < G::CHK; ++k)
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (k < G::NCH / 4 || 4 * k + t.g < G::NCH) a.acc[cbase + off(k, i)] = old[k][i] + zz[k][i];
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
    float2 old[G::CHK][4], psv[G::CHK][4];
    float vpv[G::CHK][4];
#pragma unroll
    for (int k = 0; k < G::CHK; ++k)
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (k < G::NCH / 4 || 4 * k + t.g < G::NCH) {
          old[k][i] = __ldcg(a.acc + cbase + off(k, i));
          psv[k][i] = __ldg(own + off(k, i));
          vpv[k][i] = __ldg(vpq + off(k, i));
        }
    double ov_mf = 0.0, ov_po = 0.0;
#pragma unroll
    for (int k = 0; k < G::CHK; ++k)
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (k < G::NCH / 4 || 4 * k + t.g < G::NCH) {
          const size_t gi = cbase + off(k, i);
          const float2 mf = old[k][i] + zz[k][i];
          const float2 pv = psv[k][i];
          const float2 dl = vpv[k][i] * pv;
          const float2 po = wt * mf - wu * dl;
          if (a.pout_mf) a.pout_mf[gi] = mf;
          if (a.pout) a.pout[gi] = po;
          if (a.pout_del) a.pout_del[gi] = dl;
          ov_mf += (double)pv.x * (double)mf.x + (double)pv.y * (double)mf.y;
          ov_po += (double)pv.x * (double)po.x + (double)pv.y * (double)po.y;
        }
    if (a.ovl) {
      // deterministic per-tile partial sums: warp shuffles, then thread 0
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        ov_mf += __shfl_xor_sync(0xffffffffu, ov_mf, o);
        ov_po += __shfl_xor_sync(0xffffffffu, ov_po, o);
      }
      if ((threadIdx.x & 31) == 0) {
        sh.ovr[t.warp][0] = ov_mf;
        sh.ovr[t.warp][1] = ov_po;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        double x = 0.0, y = 0.0;
        for (int w = 0; w < kHtWarps; ++w) {
          x += sh.ovr[w][0];
          y += sh.ovr[w][1];
        }
        a.ovl[((size_t)(s - a.s0) * G::T + tile) * 2 + 0] = x;
        a.ovl[((size_t)(s - a.s0) * G::T + tile) * 2 + 1] = y;
      }
    }
  }
}

template <int N>
__global__ void __launch_bounds__(kHtThreads, 1) hpsi_tc_kernel(HtArgs a) {
  using G = HtGeo<N>;
  extern __shared__ unsigned char ht_smem_raw[];
  __shared__ HtShared sh;
  unsigned char* bs = reinterpret_cast<unsigned char*>(((uintptr_t)ht_smem_raw + 1023) & ~(uintptr_t)1023);
  float2* ps = reinterpret_cast<float2*>(bs + a.bbytes);
  float4* fs = reinterpret_cast<float4*>(ps + G::PSZ);
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
  t.g = warp >> 2;
  t.row = 32 * q + lane;
  t.ln = t.row >> 1;
  t.c = t.row & 1;
  t.kp = t.c ? -1.f : 1.f;
  t.tb = sh.tmem_base;
  t.tl = t.tb + ((uint32_t)(32 * q) << 16);
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
// k sin(2 pi k (m - l) / n), kf = 2 pi / (n d)), further rows zero;
// hi = tf32(D), lo = tf32(D - hi).
template <int N>
int hpsi_tc_prepare_t(hfb_ctx_s* c) {
  using G = HtGeo<N>;
  constexpr uint32_t BALL = 3 * G::BAXIS;
  std::vector<unsigned char> img(BALL, 0);
  for (int ax = 0; ax < 3; ++ax) {
    const double kf = 2.0 * kPi / (N * c->d[ax]);
    for (int row = 0; row < G::N2; ++row)
      for (int l = 0; l < N; ++l) {
        double v = 0.0;
        if (row < N) {
          for (int k = 1; k < N / 2; ++k) {
            const int ph = (((k * (row - l)) % N) + N) % N;
            v += k * sin(2.0 * kPi * ph / N);
          }
          v *= -2.0 * kf / N;
        }
        const float hi = tf32_host((float)v);
        const float lo = tf32_host((float)(v - (double)hi));
        const size_t off = (size_t)(l / 32) * G::N2 * 128 + sw128_host(row, (l % 32) / 4) + (l % 4) * 4;
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
  const int slots = sm_count();
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

bool hpsi_tc_available(hfb_ctx_s* c, int prec) {
  return prec == HFB_F32 && c->use_tcgen05 && c->hpsi_kind != 2 && c->hpsi_b;
}

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
