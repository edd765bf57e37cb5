// Single-precision hpsi (hpsi01, meanfield.py:41-159) on the tcgen05 tensor
// cores: bf16 three-term operands, two CTAs per SM.
//
// The algebra is that of the FFT path (hpsi.cu): along each axis d
//     out_d = L_d(D psi) + D (L_d psi - B D psi) + Nyquist term,
// with D the spectral first derivative whose k = 0 and n/2 bins are zero (a
// real n x n matrix), B the effective mass, L_d the pointwise 2x2 complex
// current / spin-orbit operator of the axis (meanfield.py:63-141) and the
// Nyquist term (pi/d)^2 mean_line(B) (-1)^j sum_l (-1)^l psi_l / n.  D on
// all lines of a state is a real GEMM with K = n: per axis and tile
//     GEMM 1  e = D psi,           then pointwise o = L_d e,
//                                  w = L_d psi - B e,
//     GEMM 2  o + D w,             then the epilogue adds the Nyquist term
//                                  (and, in the z pass, the local terms).
//
// Operands.  Each fp32 value x is split into three bf16 numbers
// x = h + m + l (h = bf16(x), m = bf16(x - h), l = bf16(x - h - m); both
// differences are exact in fp32) and so is D; the six products h Dh, h Dm,
// m Dh, h Dl, m Dm, l Dh (smallest first) carry 24 significant bits, the
// dropped ones are below 2^-24 relative.  bf16 has the fp32 exponent range,
// so no scaling is needed.
//
// TMEM (256 columns per CTA): the A operand of both GEMMs, psi and then w,
// as six bf16-pair parts (h, m, l of Re and Im; K/2 columns each, 144 for
// n = 48) and one accumulator pair (Re, Im; 96 columns), which holds e,
// is overwritten with o by the pointwise step and receives D w on top.
// Nothing else is parked in TMEM: L_d psi is recomputed from psi kept in
// registers.  With 240 of 512 columns a tile, two 256-thread CTAs share an
// SM, and each one's GEMMs and memory waits overlap the other's arithmetic.
//
// Tile: 64 lines of one axis of one state = 128 GEMM rows, row = 2 line +
// spinor component.  Thread (row, half g) owns the row's points
// [g n/2, (g+1) n/2), so its TMEM accesses are whole column runs.  The
// other component of a point sits in the neighbouring lane (shuffle).
// Fields are repacked once per launch per pass into a tile-major layout
// F[tile][point][line] so that every pass reads them coalesced, with the
// line means of B precomputed for the Nyquist term.
//
// Scheduling as in the tf32 kernel (hpsi_tc.cu): persistent CTAs take tasks
// from an atomic ticket in the order [z tiles][y tiles][x tiles] per group
// of states; a y (x) tile waits before its epilogue until every z (y) tile
// of its state is published.  A CTA takes its first ticket only after its
// TMEM allocation succeeded, and tasks wait only on tickets handed out
// before their own, so the schedule cannot deadlock.  Every wait is bounded
// (the context's wait limit): a timeout latches HFB_ERR_TIMEOUT, raises an
// abort flag the other CTAs see, waits for the CTA's own MMAs and releases
// TMEM.
#include <limits.h>
#include <math.h>
#include <string.h>
#include <vector>
#include "hfb_ctx.cuh"
#include "tc_sm100.cuh"

namespace hfb {

namespace {

constexpr int kHbThreads = 256;        // 8 warps: 4 TMEM lane quarters x 2 halves of a line
constexpr int kHbWarps = kHbThreads / 32;
constexpr int kHbLines = 64;           // lines per tile (x 2 components = 128 GEMM rows)
constexpr int kHbTmemCols = 256;
constexpr long long kHbDrainLimit = 2000000000LL;   // waits for the CTA's own MMAs before exit
// dynamic shared memory per CTA is at least this, so that no third CTA can
// join two on one SM (228 KB per SM): TMEM is budgeted for two
constexpr size_t kHbMinSmem = 80 * 1024;

template <int N>
struct HbGeo {
  static constexpr int KP = ((N + 15) / 16) * 16;   // K padded to the MMA's 16
  static constexpr int N2 = ((N + 15) / 16) * 16;   // MMA N (rows of B)
  static constexpr int KS = KP / 16;                // MMA K steps
  static constexpr int ACOL = KP / 2;               // TMEM columns of one A part (bf16 pairs)
  static constexpr uint32_t DCOL = 6 * ACOL;        // accumulator Re; Im at DCOL + N2
  static constexpr int PT = N / 2;                  // points per thread
  static constexpr int NCK = PT / 4;                // 4-point chunks per thread
  static constexpr int T = N * N / kHbLines;        // tiles per state and axis
  static constexpr uint32_t BTILE = N2 * 128;       // one bf16 B tile: N2 rows of 64 bf16
  static constexpr uint32_t BAXIS = 3 * BTILE;      // h, m, l
  static_assert(DCOL + 2 * N2 <= kHbTmemCols, "TMEM budget of one tile");
  static_assert(N % 8 == 0 && (N * N) % kHbLines == 0 && N <= 48, "grid size");
  static_assert(BTILE % 1024 == 0, "B tiles stay 1024-byte aligned");
};

struct HbArgs {
  const float4* F;           // [2 iq][3 pass][n^3] pass fields, tile-major per pass
  const float4* FL;          // [2 iq][n^3] local fields, tile-major in the z-pass order
  const float* bbar;         // [2 iq][3 pass][n^2] line means of B
  const float* pot;          // [2][12][n^3] (v_pair for the x-pass epilogue)
  const float2* psi;
  float2* acc;
  const unsigned char* bmat; // [1 or 3 axes][h, m, l] bf16 B tiles
  uint32_t bstride;          // bytes between the axes' B tiles (0: one set for all axes)
  uint32_t bbytes;
  int s0, ns, nneut, group;
  float nq[3];               // (pi/d)^2 / n per axis
  const double* weight;
  const double* weightuv;
  float2* pout;
  float2* pout_mf;
  float2* pout_del;
  double* ovl;
  int* cnt;                  // [0] ticket, [1] abort, [2] never written, [3 + 2 s + p] published tiles
  int* status;
  long long wait_limit;      // clock cycles of any one bounded wait
  int probe;                 // nonzero: CTA 0 first waits on cnt[2] (the timeout path, for tests)
};

// tile-major index of point j of line L of a pass
template <int N>
__host__ __device__ __forceinline__ size_t hb_fidx(int L, int j) {
  return ((size_t)(L >> 6) * N + j) * kHbLines + (L & 63);
}

// Fields per grid point and pass (current and spin-orbit fields halved, as
// they enter L_d): x (B, aq_x/2, wl_y/2, wl_z/2), y (B, aq_y/2, wl_x/2,
// wl_z/2), z (B, aq_z/2, wl_x/2, wl_y/2); local (upot, spot_x, spot_y,
// spot_z) in the z-pass order.  Also zeroes the scheduling counters.
template <int N>
__global__ void hb_fields_kernel(const float* __restrict__ pot, float4* __restrict__ F, float4* __restrict__ FL,
                                 int* cnt, int ncnt) {
  constexpr size_t n3 = (size_t)N * N * N;
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < (size_t)ncnt) cnt[i] = 0;
  if (i >= 2 * n3) return;
  const int iq = (int)(i / n3);
  const size_t g = i - (size_t)iq * n3;
  const int x = (int)(g / (N * N)), y = (int)((g / N) % N), z = (int)(g % N);
  const float* p = pot + (size_t)iq * 12 * n3;
  const float bm = p[n3 + g];
  const float w0 = 0.5f * p[9 * n3 + g], w1 = 0.5f * p[10 * n3 + g], w2 = 0.5f * p[11 * n3 + g];
  float4* f = F + (size_t)iq * 3 * n3;
  f[hb_fidx<N>(y * N + z, x)] = make_float4(bm, 0.5f * p[3 * n3 + g], w1, w2);
  f[n3 + hb_fidx<N>(x * N + z, y)] = make_float4(bm, 0.5f * p[4 * n3 + g], w0, w2);
  f[2 * n3 + hb_fidx<N>(x * N + y, z)] = make_float4(bm, 0.5f * p[5 * n3 + g], w0, w1);
  FL[(size_t)iq * n3 + hb_fidx<N>(x * N + y, z)] = make_float4(p[g], p[6 * n3 + g], p[7 * n3 + g], p[8 * n3 + g]);
}

// First grid point of line L of axis AX (points follow at stride 1, n, n^2
// for AX = 2, 1, 0).
template <int N, int AX>
__host__ __device__ __forceinline__ size_t hb_line_base(int L) {
  return AX == 2 ? (size_t)L * N : (AX == 1 ? (size_t)(L / N) * N * N + (L % N) : (size_t)L);
}

// Line means of B for the Nyquist term: bbar[iq][AX][L]
template <int N>
__global__ void hb_bbar_kernel(const float* __restrict__ pot, float* __restrict__ bbar) {
  constexpr size_t n3 = (size_t)N * N * N;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 2 * 3 * N * N) return;
  const int iq = i / (3 * N * N), ax = (i / (N * N)) % 3, L = i % (N * N);
  const float* b = pot + ((size_t)iq * 12 + 1) * n3;
  const size_t base = ax == 2 ? hb_line_base<N, 2>(L) : (ax == 1 ? hb_line_base<N, 1>(L) : hb_line_base<N, 0>(L));
  const size_t stride = ax == 2 ? 1 : (ax == 1 ? (size_t)N : (size_t)N * N);
  float s = 0.f;
  for (int j = 0; j < N; ++j) s += b[base + j * stride];
  bbar[i] = s * (1.f / N);
}

// L_d of the own component: L_d x_c = i alpha_c x_c + (beta_c + i gamma_c)
// x_cbar with (kp = +1 upper, -1 lower component; f the pass's halved
// fields), meanfield.py:63-141:
//   z: alpha = -aq_z/2,               beta = kp wl_x/2,  gamma = -wl_y/2
//   y: alpha = -(aq_y + kp wl_x)/2,   beta = 0,          gamma = wl_z/2
//   x: alpha = -(aq_x - kp wl_y)/2,   beta = -kp wl_z/2, gamma = 0
template <int AX>
__device__ __forceinline__ float2 hb_l(float4 f, float kp, float2 a, float2 b) {
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

// bf16 pair {x0 in the low half, x1 in the high half}, round to nearest
__device__ __forceinline__ uint32_t hb_pack(float x0, float x1) {
  uint32_t r;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(x1), "f"(x0));
  return r;
}
__device__ __forceinline__ float hb_lo(uint32_t p) { return __uint_as_float(p << 16); }
__device__ __forceinline__ float hb_hi(uint32_t p) { return __uint_as_float(p & 0xffff0000u); }

// x0, x1 -> three bf16 pairs h, m, l with x = h + m + l to 2^-24
__device__ __forceinline__ void hb_split3(float x0, float x1, uint32_t& h, uint32_t& m, uint32_t& l) {
  h = hb_pack(x0, x1);
  const float r0 = x0 - hb_lo(h), r1 = x1 - hb_hi(h);
  m = hb_pack(r0, r1);
  l = hb_pack(r0 - hb_lo(m), r1 - hb_hi(m));
}

// A operand parts: 0 h Re, 1 h Im, 2 m Re, 3 m Im, 4 l Re, 5 l Im.  Store
// the split of 4 points (v0..v3) at this thread's column ``col`` (even).
template <int N>
__device__ __forceinline__ void hb_store_a(uint32_t tl, int col, float2 v0, float2 v1, float2 v2, float2 v3) {
  using G = HbGeo<N>;
  uint32_t h0, m0, l0, h1, m1, l1;
  hb_split3(v0.x, v1.x, h0, m0, l0);
  hb_split3(v2.x, v3.x, h1, m1, l1);
  tc::tmem_st_x2(tl + 0 * G::ACOL + col, h0, h1);
  tc::tmem_st_x2(tl + 2 * G::ACOL + col, m0, m1);
  tc::tmem_st_x2(tl + 4 * G::ACOL + col, l0, l1);
  hb_split3(v0.y, v1.y, h0, m0, l0);
  hb_split3(v2.y, v3.y, h1, m1, l1);
  tc::tmem_st_x2(tl + 1 * G::ACOL + col, h0, h1);
  tc::tmem_st_x2(tl + 3 * G::ACOL + col, m0, m1);
  tc::tmem_st_x2(tl + 5 * G::ACOL + col, l0, l1);
}

// (D Re, D Im) (+)= A B^T over the six bf16 products, smallest first, each
// over the K steps
template <int N>
__device__ __forceinline__ void hb_gemm(uint32_t tb, uint32_t bsm, bool accumulate) {
  using G = HbGeo<N>;
  constexpr uint32_t idesc = tc::idesc_bf16(128, G::N2);
  constexpr int ap[6] = {4, 2, 0, 2, 0, 0};   // A part (Re; Im is the next part)
  constexpr int bp[6] = {0, 1, 2, 0, 1, 0};   // B tile: 0 h, 1 m, 2 l
  bool first = !accumulate;
#pragma unroll
  for (int t = 0; t < 6; ++t)
#pragma unroll
    for (int ks = 0; ks < G::KS; ++ks) {
      const uint64_t bd = tc::sw128_desc(bsm + bp[t] * G::BTILE + ks * 32);
      const uint32_t acc = first ? 0u : 1u;
      tc::mma_f16_ta(tb + G::DCOL, tb + ap[t] * G::ACOL + ks * 8, bd, idesc, acc);
      tc::mma_f16_ta(tb + G::DCOL + G::N2, tb + (ap[t] + 1) * G::ACOL + ks * 8, bd, idesc, acc);
      first = false;
    }
}

// Wait until *cnt >= target (acquire); false on abort or timeout.
__device__ __forceinline__ bool hb_wait_count(const int* cnt, const int* abort_flag, int target, long long limit) {
  const long long t0 = clock64();
  for (;;) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(cnt) : "memory");
    if (v >= target) return true;
    if (*(const volatile int*)abort_flag) return false;
    if (clock64() - t0 > limit) return false;
    __nanosleep(64);
  }
}

struct HbThread {
  int row, ln, c, g, warp, j0, c0;
  uint32_t tb, tl;
  float kp;
};

struct HbShared {
  uint64_t bar_b, bar_mma;
  uint32_t tmem_base;
  int task, next, bad;
  float2 alt[128][2];          // partial alternating sums per row and half
  double ovr[kHbWarps][2];
};

// Next ticket (INT_MAX once another CTA has aborted).
__device__ __forceinline__ int hb_ticket(const HbArgs& a) {
  int k = atomicAdd(a.cnt, 1);
  if (*(volatile int*)(a.cnt + 1)) k = INT_MAX;
  return k;
}

// Task -> (pass, state, tile); tasks run [z tiles][y tiles][x tiles] per
// group of ``group`` states.  False past the last task.
template <int N>
__device__ __forceinline__ bool hb_decode(const HbArgs& a, int task, int& pass, int& s, int& tile) {
  constexpr int T = HbGeo<N>::T;
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

// The thread's PT points of its row, complex, from a state-sized array
template <int N, int AX>
__device__ __forceinline__ void hb_load_row(const float2* __restrict__ src, size_t cb, float2 (&v)[HbGeo<N>::PT]) {
  using G = HbGeo<N>;
  constexpr size_t STRIDE = AX == 2 ? 1 : (AX == 1 ? (size_t)N : (size_t)N * N);
  if (AX == 2) {
    const float4* s4 = reinterpret_cast<const float4*>(src + cb);   // cb even: 16-byte aligned
#pragma unroll
    for (int i = 0; i < G::PT / 2; ++i) {
      const float4 q = __ldg(s4 + i);
      v[2 * i] = make_float2(q.x, q.y);
      v[2 * i + 1] = make_float2(q.z, q.w);
    }
  } else {
#pragma unroll
    for (int i = 0; i < G::PT; ++i) v[i] = __ldg(src + cb + i * STRIDE);
  }
}

// Points 4k .. 4k+3 of the thread's run
template <int N, int AX>
__device__ __forceinline__ void hb_load_chunk(const float2* __restrict__ src, size_t cb, int k, float2 (&v)[4]) {
  constexpr size_t STRIDE = AX == 2 ? 1 : (AX == 1 ? (size_t)N : (size_t)N * N);
  if (AX == 2) {
    const float4* s4 = reinterpret_cast<const float4*>(src + cb) + 2 * k;
    const float4 q0 = __ldg(s4), q1 = __ldg(s4 + 1);
    v[0] = make_float2(q0.x, q0.y);
    v[1] = make_float2(q0.z, q0.w);
    v[2] = make_float2(q1.x, q1.y);
    v[3] = make_float2(q1.z, q1.w);
  } else {
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i] = __ldg(src + cb + (4 * k + i) * STRIDE);
  }
}

template <int N, int AX, int P>
__device__ __forceinline__ void hb_tile(const HbArgs& a, const HbThread& t, HbShared& sh, uint32_t bsm, int s,
                                        int tile, uint32_t& phase, bool& b_ready) {
  using G = HbGeo<N>;
  constexpr size_t N3 = (size_t)N * N * N;
  constexpr size_t STRIDE = AX == 2 ? 1 : (AX == 1 ? (size_t)N : (size_t)N * N);
  const int iq = s >= a.nneut ? 1 : 0;
  const int L = tile * kHbLines + t.ln;
  const size_t cb = ((size_t)s * 2 + t.c) * N3 + hb_line_base<N, AX>(L) + (size_t)t.j0 * STRIDE;
  const uint32_t bax = bsm + AX * a.bstride;

  // ---- staging: psi -> the A operand; partial alternating sums
  {
    float2 v[G::PT];
    hb_load_row<N, AX>(a.psi, cb, v);
    float2 alt = make_float2(0.f, 0.f);
#pragma unroll
    for (int i = 0; i < G::PT; ++i) {
      alt.x += (i & 1) ? -v[i].x : v[i].x;   // (-1)^j psi_j, j0 even
      alt.y += (i & 1) ? -v[i].y : v[i].y;
    }
    sh.alt[t.row][t.g] = alt;
#pragma unroll
    for (int k = 0; k < G::NCK; ++k)
      hb_store_a<N>(t.tl, t.c0 + 2 * k, v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
  }
  tc::tmem_st_wait();
  tc::fence_before();
  __syncthreads();
  // The pointwise step's first global inputs do not depend on GEMM 1:
  // they are loaded while it runs.
  const float4* fp = a.F + ((size_t)iq * 3 + AX) * N3 + hb_fidx<N>(L, t.j0);
  float4 fn[4];
  float2 pn[4];
  hb_load_chunk<N, AX>(a.psi, cb, 0, pn);
#pragma unroll
  for (int i = 0; i < 4; ++i) fn[i] = __ldg(fp + i * kHbLines);
  // ---- GEMM 1: e = D psi
  if (threadIdx.x == 0) {
    tc::fence_after();
    if (!b_ready) {
      // on a timeout b_ready stays false: the exit path waits for the copy
      if (tc::mbar_wait(&sh.bar_b, 0, a.wait_limit)) b_ready = true;
      else sh.bad = 1;
    }
    if (!sh.bad) {
      hb_gemm<N>(t.tb, bax, false);
      tc::mma_commit(&sh.bar_mma);
      if (!tc::mbar_wait(&sh.bar_mma, phase & 1, a.wait_limit)) sh.bad = 1;
    }
  }
  ++phase;
  __syncthreads();
  if (sh.bad) return;
  tc::fence_after();
  const float2 alt = make_float2(sh.alt[t.row][0].x + sh.alt[t.row][1].x, sh.alt[t.row][0].y + sh.alt[t.row][1].y);

  // ---- pointwise: o = L_d e over e in the accumulator, w = L_d psi - B e into A.
  // The global loads of chunk k + 1 are issued before the TMEM accesses of
  // chunk k (which the compiler cannot reorder memory operations across),
  // so they are in flight while chunk k is computed.
#pragma unroll
  for (int k = 0; k < G::NCK; ++k) {
    float4 f[4];
    float2 pc[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      f[i] = fn[i];
      pc[i] = pn[i];
    }
    if (k + 1 < G::NCK) {
      hb_load_chunk<N, AX>(a.psi, cb, k + 1, pn);
#pragma unroll
      for (int i = 0; i < 4; ++i) fn[i] = __ldg(fp + (4 * (k + 1) + i) * kHbLines);
    }
    uint32_t er[4], em[4];
    tc::tmem_ld_x4(t.tl + G::DCOL + t.j0 + 4 * k, er);
    tc::tmem_ld_x4(t.tl + G::DCOL + G::N2 + t.j0 + 4 * k, em);
    tc::tmem_ld_wait();
    uint32_t orr[4], om[4];
    float2 w[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float2 ev = make_float2(__uint_as_float(er[i]), __uint_as_float(em[i]));
      const float2 eo = make_float2(__shfl_xor_sync(0xffffffffu, ev.x, 1), __shfl_xor_sync(0xffffffffu, ev.y, 1));
      const float2 pv = pc[i];
      const float2 po = make_float2(__shfl_xor_sync(0xffffffffu, pv.x, 1), __shfl_xor_sync(0xffffffffu, pv.y, 1));
      const float2 o = hb_l<AX>(f[i], t.kp, ev, eo);
      const float2 n = hb_l<AX>(f[i], t.kp, pv, po);
      w[i] = make_float2(n.x - f[i].x * ev.x, n.y - f[i].x * ev.y);
      orr[i] = __float_as_uint(o.x);
      om[i] = __float_as_uint(o.y);
    }
    tc::tmem_st_x4(t.tl + G::DCOL + t.j0 + 4 * k, orr);
    tc::tmem_st_x4(t.tl + G::DCOL + G::N2 + t.j0 + 4 * k, om);
    hb_store_a<N>(t.tl, t.c0 + 2 * k, w[0], w[1], w[2], w[3]);
  }
  tc::tmem_st_wait();
  tc::fence_before();
  __syncthreads();
  // ---- GEMM 2: o + D w; a y (x) tile then waits for the z (y) pass of its state
  if (threadIdx.x == 0) {
    tc::fence_after();
    hb_gemm<N>(t.tb, bax, true);
    tc::mma_commit(&sh.bar_mma);
    if (P > 0 && !hb_wait_count(a.cnt + 3 + 2 * (s - a.s0) + (P - 1), a.cnt + 1, G::T, a.wait_limit)) {
      sh.bad = 1;
      latch_error(a.status, HFB_ERR_TIMEOUT);
      atomicExch(a.cnt + 1, 1);
    }
  }
  __syncthreads();   // the previous pass of the state is complete in memory

  // ---- epilogue: o + D w + Nyquist term, 4 points at a time.  The global
  // inputs of chunk k + 1 are loaded before the TMEM reads of chunk k (as in
  // the pointwise step), chunk 0's while GEMM 2 runs: the previous pass's
  // sum (y, x passes), psi and the local fields for the z pass's upot / spin
  // terms, psi and v_pair for the x pass's outputs.
  const float nyq = a.nq[AX] * a.bbar[((size_t)iq * 3 + AX) * N * N + L];
  const float wt = (P == 2 && a.weight) ? (float)a.weight[s] : 1.f;
  const float wu = (P == 2 && a.weightuv) ? (float)a.weightuv[s] : 0.f;
  const float* vpq = a.pot + ((size_t)iq * 12 + 2) * N3 + hb_line_base<N, AX>(L) + (size_t)t.j0 * STRIDE;
  const float4* flp = a.FL + (size_t)iq * N3 + hb_fidx<N>(L, t.j0);
  double ov_mf = 0.0, ov_po = 0.0;
  float2 qn[4], on[4];
  float4 gn[4];
  float vn[4];
  auto fetch = [&](int k, float2 (&pc)[4], float2 (&od)[4], float4 (&gl)[4], float (&vp)[4]) {
    if (P != 1) hb_load_chunk<N, AX>(a.psi, cb, k, pc);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      if (P > 0) od[i] = __ldcg(a.acc + cb + (4 * k + i) * STRIDE);
      if (P == 0) gl[i] = __ldg(flp + (4 * k + i) * kHbLines);
      if (P == 2) vp[i] = __ldg(vpq + (4 * k + i) * STRIDE);
    }
  };
  if (!sh.bad) fetch(0, qn, on, gn, vn);
  if (threadIdx.x == 0 && !tc::mbar_wait(&sh.bar_mma, phase & 1, a.wait_limit)) sh.bad = 1;
  ++phase;
  __syncthreads();
  if (sh.bad) return;
  tc::fence_after();
#pragma unroll
  for (int k = 0; k < G::NCK; ++k) {
    float2 pc[4], old[4];
    float4 gl[4];
    float vp[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      pc[i] = qn[i];
      old[i] = on[i];
      gl[i] = gn[i];
      vp[i] = vn[i];
    }
    if (k + 1 < G::NCK) fetch(k + 1, qn, on, gn, vn);
    uint32_t dr[4], di[4];
    tc::tmem_ld_x4(t.tl + G::DCOL + t.j0 + 4 * k, dr);
    tc::tmem_ld_x4(t.tl + G::DCOL + G::N2 + t.j0 + 4 * k, di);
    tc::tmem_ld_wait();
    float2 z[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float sg = (i & 1) ? -nyq : nyq;   // (-1)^j, j0 even
      z[i] = make_float2(__uint_as_float(dr[i]) + sg * alt.x, __uint_as_float(di[i]) + sg * alt.y);
      if (P == 0) {
        // upot psi + sigma.spot psi (meanfield.py:47-58), with the other
        // spinor component from the neighbouring lane
        const float2 pv = pc[i];
        const float2 po = make_float2(__shfl_xor_sync(0xffffffffu, pv.x, 1), __shfl_xor_sync(0xffffffffu, pv.y, 1));
        const float d = gl[i].x + t.kp * gl[i].w, s1 = t.kp * gl[i].z;
        z[i].x += d * pv.x + gl[i].y * po.x + s1 * po.y;
        z[i].y += d * pv.y + gl[i].y * po.y - s1 * po.x;
      }
    }
    if (P == 0) {
      float4* d4 = reinterpret_cast<float4*>(a.acc + cb) + 2 * k;
      d4[0] = make_float4(z[0].x, z[0].y, z[1].x, z[1].y);
      d4[1] = make_float4(z[2].x, z[2].y, z[3].x, z[3].y);
    } else if (P == 1) {
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int j = 4 * k + i;
        a.acc[cb + j * STRIDE] = make_float2(old[i].x + z[i].x, old[i].y + z[i].y);
      }
    } else {
      // x pass: h psi complete; weights, v_pair psi, overlaps
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int j = 4 * k + i;
        const size_t gi = cb + j * STRIDE;
        const float2 mf = make_float2(old[i].x + z[i].x, old[i].y + z[i].y);
        const float2 pv = pc[i];
        const float2 dl = make_float2(vp[i] * pv.x, vp[i] * pv.y);
        const float2 po = make_float2(wt * mf.x - wu * dl.x, wt * mf.y - wu * dl.y);
        if (a.pout_mf) a.pout_mf[gi] = mf;
        if (a.pout) a.pout[gi] = po;
        if (a.pout_del) a.pout_del[gi] = dl;
        ov_mf += (double)pv.x * (double)mf.x + (double)pv.y * (double)mf.y;
        ov_po += (double)pv.x * (double)po.x + (double)pv.y * (double)po.y;
      }
    }
  }
  tc::fence_before();   // accumulator reads done before the next tile's GEMM 1
  if (P == 2 && a.ovl) {
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
      for (int w = 0; w < kHbWarps; ++w) {
        x += sh.ovr[w][0];
        y += sh.ovr[w][1];
      }
      a.ovl[((size_t)(s - a.s0) * G::T + tile) * 2 + 0] = x;
      a.ovl[((size_t)(s - a.s0) * G::T + tile) * 2 + 1] = y;
    }
  }
  if (P < 2) {
    // publish this tile for the next pass of the state
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(a.cnt + 3 + 2 * (s - a.s0) + P, 1);
    }
  }
}

template <int N>
__global__ void __launch_bounds__(kHbThreads, 2) hpsi_bf3_kernel(HbArgs a) {
  using G = HbGeo<N>;
  extern __shared__ unsigned char hb_smem_raw[];
  __shared__ HbShared sh;
  unsigned char* bs = reinterpret_cast<unsigned char*>(((uintptr_t)hb_smem_raw + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) {
    tc::tmem_alloc(&sh.tmem_base, kHbTmemCols);
    tc::tmem_relinquish();
  }
  if (tid == 0) {
    sh.bad = 0;
    tc::mbar_init(&sh.bar_b, 1);
    tc::mbar_init(&sh.bar_mma, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    tc::mbar_arrive_expect_tx(&sh.bar_b, a.bbytes);
    tc::bulk_g2s(bs, a.bmat, a.bbytes, &sh.bar_b);
    // the timeout path, for tests: a bounded wait on a word nothing writes,
    // before this CTA holds any ticket
    if (a.probe && blockIdx.x == 0 && !hb_wait_count(a.cnt + 2, a.cnt + 1, 1, a.wait_limit)) {
      sh.bad = 1;
      latch_error(a.status, HFB_ERR_TIMEOUT);
      atomicExch(a.cnt + 1, 1);
    }
    sh.task = sh.bad ? INT_MAX : hb_ticket(a);
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();

  HbThread t;
  t.warp = warp;
  const int q = warp & 3;
  t.g = warp >> 2;
  t.row = 32 * q + lane;
  t.ln = t.row >> 1;
  t.c = t.row & 1;
  t.kp = t.c ? -1.f : 1.f;
  t.j0 = t.g * G::PT;
  t.c0 = t.g * (G::PT / 2);
  t.tb = sh.tmem_base;
  t.tl = t.tb + ((uint32_t)(32 * q) << 16);
  const uint32_t bsm = tc::smem_u32(bs);
  // K padding of the A operand (n = 24, 40): zero once, never written again
  if (G::KP > N && t.g == 1) {
#pragma unroll
    for (int p = 0; p < 6; ++p)
#pragma unroll
      for (int cpad = N / 2; cpad < G::KP / 2; cpad += 2) tc::tmem_st_x2(t.tl + p * G::ACOL + cpad, 0u, 0u);
    tc::tmem_st_wait();
  }

  uint32_t phase = 0;
  bool b_ready = false;
  int task = sh.task;
  for (;;) {
    int pass, s, tile;
    if (sh.bad || !hb_decode<N>(a, task, pass, s, tile)) break;
    if (tid == 0) sh.next = hb_ticket(a);
    if (pass == 0)
      hb_tile<N, 2, 0>(a, t, sh, bsm, s, tile, phase, b_ready);
    else if (pass == 1)
      hb_tile<N, 1, 1>(a, t, sh, bsm, s, tile, phase, b_ready);
    else
      hb_tile<N, 0, 2>(a, t, sh, bsm, s, tile, phase, b_ready);
    // every thread reads sh.next (written before the tile's first barrier)
    // before this barrier, and thread 0 rewrites it only after it
    task = sh.next;
    __syncthreads();   // sh.bad is visible; the tile's accumulator reads are done
  }
  tc::fence_before();
  __syncthreads();
  if (tid == 0) {
    if (sh.bad) {
      latch_error(a.status, HFB_ERR_TIMEOUT);
      atomicExch(a.cnt + 1, 1);
      // let this CTA's own MMAs and the B copy finish before TMEM goes
      if (phase > 0) tc::mbar_wait(&sh.bar_mma, (phase - 1) & 1, kHbDrainLimit);
    }
    if (!b_ready) tc::mbar_wait(&sh.bar_b, 0, kHbDrainLimit);
  }
  __syncthreads();
  if (warp == 0) {
    tc::fence_after();
    tc::tmem_dealloc(t.tb, kHbTmemCols);
  }
}

// bf16 round to nearest even of a finite double (through float)
uint16_t bf16_host(double x) {
  const float f = (float)x;
  uint32_t u;
  memcpy(&u, &f, 4);
  u += 0x7fffu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}
double bf16_value(uint16_t b) {
  const uint32_t u = (uint32_t)b << 16;
  float f;
  memcpy(&f, &u, 4);
  return (double)f;
}

uint32_t hb_sw128_host(int r, int c) { return (uint32_t)((r >> 3) * 1024 + (r & 7) * 128 + ((c ^ (r & 7)) << 4)); }

// B tiles of the three axes: row m < n holds D[m][:] (the spectral first
// derivative with the k = 0 and n/2 bins zeroed, -(2 kf / n) sum_{k=1}^{n/2-1}
// k sin(2 pi k (m - l) / n), kf = 2 pi / (n d)), further rows and K columns
// zero; split D = h + m + l in bf16.
template <int N>
int hpsi_bf3_prepare_t(hfb_ctx_s* c) {
  using G = HbGeo<N>;
  constexpr uint32_t BALL = 3 * G::BAXIS;
  std::vector<unsigned char> img(BALL, 0);
  for (int ax = 0; ax < 3; ++ax) {
    const double kf = 2.0 * kPi / (N * c->d[ax]);
    for (int row = 0; row < N; ++row)
      for (int l = 0; l < N; ++l) {
        double v = 0.0;
        for (int k = 1; k < N / 2; ++k) {
          const int ph = (((k * (row - l)) % N) + N) % N;
          v += k * sin(2.0 * kPi * ph / N);
        }
        v *= -2.0 * kf / N;
        const uint16_t h = bf16_host(v);
        const double r1 = v - bf16_value(h);
        const uint16_t m = bf16_host(r1);
        const uint16_t lo = bf16_host(r1 - bf16_value(m));
        const size_t off = hb_sw128_host(row, l / 8) + (l % 8) * 2;
        memcpy(&img[ax * G::BAXIS + 0 * G::BTILE + off], &h, 2);
        memcpy(&img[ax * G::BAXIS + 1 * G::BTILE + off], &m, 2);
        memcpy(&img[ax * G::BAXIS + 2 * G::BTILE + off], &lo, 2);
      }
  }
  if (cudaMalloc(&c->hpsi_bf3_b, BALL) != cudaSuccess) {
    cudaGetLastError();
    c->hpsi_bf3_b = nullptr;
    return HFB_ERR_ALLOC;
  }
  if (cudaMemcpy(c->hpsi_bf3_b, img.data(), BALL, cudaMemcpyHostToDevice) != cudaSuccess) return HFB_ERR_CUDA;
  return HFB_OK;
}

int hb_sm_count() {
  static const int n = [] {
    int d = 0, v = 0;
    cudaGetDevice(&d);
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, d);
    return v > 0 ? v : 1;
  }();
  return n;
}

template <int N>
int hpsi_bf3_launch_t(hfb_ctx_s* c, const void* pot, int s0, int ns, int nneut, const void* psi,
                      const double* weight, const double* weightuv, void* acc, void* pout, void* pout_mf,
                      void* pout_del, double* ovl, cudaStream_t st) {
  using G = HbGeo<N>;
  constexpr size_t N3 = (size_t)N * N * N;
  const size_t fbytes = sizeof(float4) * 8 * N3;            // F (6 n^3) + FL (2 n^3)
  const size_t bbytes_bar = sizeof(float) * 6 * N * N;
  const int ncnt = 3 + 2 * ns;
  unsigned char* scr =
      (unsigned char*)scratch(c, hfb_ctx_s::S_HPT, fbytes + bbytes_bar + sizeof(int) * (size_t)ncnt);
  if (!scr) return HFB_ERR_ALLOC;
  float4* F = reinterpret_cast<float4*>(scr);
  float4* FL = F + 6 * N3;
  float* bbar = reinterpret_cast<float*>(scr + fbytes);
  int* cnt = reinterpret_cast<int*>(scr + fbytes + bbytes_bar);
  const size_t tot = 2 * N3 > (size_t)ncnt ? 2 * N3 : (size_t)ncnt;
  hb_fields_kernel<N><<<(unsigned)((tot + 255) / 256), 256, 0, st>>>((const float*)pot, F, FL, cnt, ncnt);
  HFB_CHECK_LAUNCH();
  hb_bbar_kernel<N><<<(6 * N * N + 255) / 256, 256, 0, st>>>((const float*)pot, bbar);
  HFB_CHECK_LAUNCH();
  const int slots = 2 * hb_sm_count();
  int group = (slots + G::T / 2) / G::T;
  if (group < 1) group = 1;
  if (group > ns) group = ns;
  const int ntask = 3 * ns * G::T;
  HbArgs a;
  a.F = F;
  a.FL = FL;
  a.bbar = bbar;
  a.pot = (const float*)pot;
  a.psi = (const float2*)psi;
  a.acc = (float2*)acc;
  a.bmat = c->hpsi_bf3_b;
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
  a.wait_limit = c->wait_limit;
  a.probe = c->timeout_probe;
  c->timeout_probe = 0;   // one launch only
  size_t smem = (size_t)a.bbytes + 1024;
  if (smem < kHbMinSmem) smem = kHbMinSmem;
  allow_max_dynamic_smem(hpsi_bf3_kernel<N>);
  hpsi_bf3_kernel<N><<<ntask < slots ? ntask : slots, kHbThreads, smem, st>>>(a);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

}  // namespace

int hpsi_bf3_prepare(hfb_ctx_s* c) {
  c->hpsi_bf3_b = nullptr;
  switch (c->n) {
    case 24: return hpsi_bf3_prepare_t<24>(c);
    case 32: return hpsi_bf3_prepare_t<32>(c);
    case 40: return hpsi_bf3_prepare_t<40>(c);
    case 48: return hpsi_bf3_prepare_t<48>(c);
    default: return HFB_OK;   // other grids keep the FFT path
  }
}

bool hpsi_bf3_available(hfb_ctx_s* c, int prec) {
  return prec == HFB_F32 && c->use_tcgen05 && c->hpsi_kind == 0 && c->hpsi_bf3_b;
}

int hpsi_bf3_parts(hfb_ctx_s* c) { return c->n * c->n / kHbLines; }

int hpsi_bf3_launch(hfb_ctx_s* c, const void* pot, int s0, int ns, int nneut, const void* psi, const double* weight,
                    const double* weightuv, void* acc, void* pout, void* pout_mf, void* pout_del, double* ovl,
                    cudaStream_t st) {
  if (ns <= 0) return HFB_OK;
  switch (c->n) {
    case 24: return hpsi_bf3_launch_t<24>(c, pot, s0, ns, nneut, psi, weight, weightuv, acc, pout, pout_mf, pout_del, ovl, st);
    case 32: return hpsi_bf3_launch_t<32>(c, pot, s0, ns, nneut, psi, weight, weightuv, acc, pout, pout_mf, pout_del, ovl, st);
    case 40: return hpsi_bf3_launch_t<40>(c, pot, s0, ns, nneut, psi, weight, weightuv, acc, pout, pout_mf, pout_del, ovl, st);
    case 48: return hpsi_bf3_launch_t<48>(c, pot, s0, ns, nneut, psi, weight, weightuv, acc, pout, pout_mf, pout_del, ovl, st);
    default: return HFB_ERR_UNSUPPORTED_GRID;
  }
}

}  // namespace hfb
