// Double-precision hpsi (hpsi01, meanfield.py:41-159) on the FP64 tensor
// cores (mma.sync m8n8k4 .f64).
//
// The algebra is the matrix form of the FFT path (hpsi.cu): along each axis d
//     out_d = L_d(D x) + D(L_d x - B D x) + Nyquist term,
// D the real n x n first-derivative matrix with its k = 0 and n/2 bins zero,
// B the effective mass, L_d the pointwise 2x2 current / spin-orbit operator
// of the axis and the Nyquist term (pi/d)^2 mean_line(B) (-1)^j
// sum_l (-1)^l x_l / n of cderv02 (levels.py:314-330).  D on the N lines of
// a staged plane is a real GEMM, D (N x N) times the plane's values (N
// points x N lines x 2 spinor components x re/im), run as 8 x 8 x 4 FP64
// MMAs: an MMA tile is 8 points x 4 lines x re/im, with both spinor
// components in two accumulators, so after GEMM 1 a thread holds e for one
// point and line in both components -- what the pointwise step needs.  w =
// L_d x - B e goes to a second plane buffer for GEMM 2; the thread's own
// tiles come back from GEMM 2 in the same positions.
//
// Kernels as in the FFT path: A (one CTA per state and x-plane) runs the z
// lines with the local upot / spin terms and then the y lines, accumulating
// in global memory (L2-resident between passes); B (one CTA per state and
// y-plane) runs the x lines and the final weights and overlaps.  The
// derivative matrices (one per axis) are built in double on the host at
// context creation.
#include <math.h>
#include <vector>
#include "hfb_ctx.cuh"
#include "hpsi.cuh"

namespace hfb {

namespace {

constexpr int kHdWarps = 8;
constexpr int kHdThreads = 32 * kHdWarps;

template <int N>
struct HdGeo {
  static constexpr int LD = N + 4;                     // complex elements per staged row (rows half a bank set apart)
  static constexpr int MB = N / 8;                     // 8-point blocks of a line
  static constexpr int LG = N / 8;                     // 8-line groups of a plane
  static constexpr int NT = MB * LG;                   // MMA tiles per pass
  static constexpr int TMAX = (NT + kHdWarps - 1) / kHdWarps;
  static constexpr int KS = N / 4;                     // k steps
  static constexpr size_t PLANE = (size_t)2 * N * LD;  // complex elements of one staged plane
  static constexpr int DLD = N + 4;                    // row stride of a staged D: rows 8 banks apart
  // plane, w buffer, alternating sums [2][N]; two derivative matrices, line means of B
  static constexpr size_t SMEM = sizeof(double2) * (2 * PLANE + 2 * N) + sizeof(double) * (2 * (size_t)N * DLD + N);
  static_assert(N % 8 == 0, "grid size");
};

__device__ __forceinline__ void hd_mma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// Staged plane buf[c][a][b] (row stride LD); a "line" of the pass runs along
// b (ROW) or along a, and pt is the position along it.
template <int N, bool ROW>
__device__ __forceinline__ int hd_at(int c, int line, int pt) {
  using G = HdGeo<N>;
  return ROW ? (c * N + line) * G::LD + pt : (c * N + pt) * G::LD + line;
}

}  // namespace

namespace {

template <int N>
constexpr int hd_dld() { return HdGeo<N>::DLD; }

// One axis pass over the N lines of the staged plane X: emits the axis's
// contribution to h x at every point of the plane, both spinor components,
// through emit(line, j, g, out0, out1, pre(g)) (g the point's index in the
// state; pre's global loads are issued before the tile's GEMM 2 MMAs).
// Dm is D for the axis (row stride hd_dld), W a second plane buffer, alt and
// bbar per-line scratch; lines start at base + line * sa (ROW) or base +
// line * sb, points are sb (ROW) or sa apart.  Ends with a CTA barrier.
template <int N, int AXIS, bool ROW, bool LOCAL, class Pre, class Emit>
__device__ __forceinline__ void hd_pass(const double2* X, double2* W, const double* Dm, double2* alt, double* bbar,
                                        const double* pot, size_t base, size_t sa, size_t sb, double nq, Pre&& pre,
                                        Emit&& emit) {
  using G = HdGeo<N>;
  constexpr size_t N3 = (size_t)N * N * N;
  constexpr int DLD = hd_dld<N>();
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  auto gidx = [&](int line, int j) -> size_t {
    return ROW ? base + (size_t)line * sa + (size_t)j * sb : base + (size_t)j * sa + (size_t)line * sb;
  };
  // Nyquist ingredients per line (levels.py:314-330): sum_l (-1)^l x_l of
  // both components and the line mean of B; one warp per line, lanes over
  // the points, a fixed shuffle tree
  for (int line = warp; line < N; line += kHdWarps) {
    double ax0 = 0.0, ay0 = 0.0, ax1 = 0.0, ay1 = 0.0, bs = 0.0;
    for (int l = lane; l < N; l += 32) {
      const double sgn = (l & 1) ? -1.0 : 1.0;
      const double2 v0 = X[hd_at<N, ROW>(0, line, l)], v1 = X[hd_at<N, ROW>(1, line, l)];
      ax0 += sgn * v0.x;
      ay0 += sgn * v0.y;
      ax1 += sgn * v1.x;
      ay1 += sgn * v1.y;
      bs += pot[1 * N3 + gidx(line, l)];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      ax0 += __shfl_xor_sync(0xffffffffu, ax0, o);
      ay0 += __shfl_xor_sync(0xffffffffu, ay0, o);
      ax1 += __shfl_xor_sync(0xffffffffu, ax1, o);
      ay1 += __shfl_xor_sync(0xffffffffu, ay1, o);
      bs += __shfl_xor_sync(0xffffffffu, bs, o);
    }
    if (lane == 0) {
      alt[line] = make_double2(ax0, ay0);
      alt[N + line] = make_double2(ax1, ay1);
      bbar[line] = bs / N;
    }
  }
  // Tile: 8 points x 8 lines.  MMA fragments: A = D row j0 + lane/4, k =
  // lane%4; B = line l0 + lane/4 at point k, one MMA each for the re and im
  // parts of the two spinor components (one double2 load gives both parts);
  // C = point j0 + lane/4, lines l0 + 2 (lane%4) + {0, 1}.
  const double h = 0.5;
  double2 o[G::TMAX][2][2];   // [tile][line of the pair][component]
  // ---- GEMM 1: e = D x, then o = L_d e (+ local terms), w = L_d x - B e
#pragma unroll
  for (int ti = 0; ti < G::TMAX; ++ti) {
    const int t = warp + ti * kHdWarps;
    if (t < G::NT) {
      const int j0 = (t / G::LG) * 8, l0 = (t % G::LG) * 8;
      const int j = j0 + (lane >> 2), lp = l0 + 2 * (lane & 3);
      // this tile's pointwise inputs are loaded before its MMAs, which hide
      // their latency
      double bm[2], aqd[2], w0[2], w1[2], w2[2], up[2], s0[2], s1[2], s2[2];
      size_t g[2];
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        g[u] = gidx(lp + u, j);
        bm[u] = pot[1 * N3 + g[u]];
        aqd[u] = pot[(3 + AXIS) * N3 + g[u]];
        w0[u] = pot[9 * N3 + g[u]];
        w1[u] = pot[10 * N3 + g[u]];
        w2[u] = pot[11 * N3 + g[u]];
        up[u] = LOCAL ? pot[g[u]] : 0.0;
        s0[u] = LOCAL ? pot[6 * N3 + g[u]] : 0.0;
        s1[u] = LOCAL ? pot[7 * N3 + g[u]] : 0.0;
        s2[u] = LOCAL ? pot[8 * N3 + g[u]] : 0.0;
      }
      double acc[4][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
      for (int ks = 0; ks < G::KS; ++ks) {
        const int pt = ks * 4 + (lane & 3);
        const double a = Dm[(j0 + (lane >> 2)) * DLD + pt];
        const double2 x0 = X[hd_at<N, ROW>(0, l0 + (lane >> 2), pt)];
        const double2 x1 = X[hd_at<N, ROW>(1, l0 + (lane >> 2), pt)];
        hd_mma(acc[0], a, x0.x);
        hd_mma(acc[1], a, x0.y);
        hd_mma(acc[2], a, x1.x);
        hd_mma(acc[3], a, x1.y);
      }
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int line = lp + u;
        const double2 e0 = make_double2(acc[0][u], acc[1][u]), e1 = make_double2(acc[2][u], acc[3][u]);
        const double2 a0 = X[hd_at<N, ROW>(0, line, j)], a1 = X[hd_at<N, ROW>(1, line, j)];
        double2 q0, q1, n0, n1;
        if (LOCAL) {
          // upot psi + sigma.spot psi (meanfield.py:47-58)
          q0 = (up[u] + s2[u]) * a0 + cmulri(s0[u], -s1[u], a1);
          q1 = (up[u] - s2[u]) * a1 + cmulri(s0[u], s1[u], a0);
        } else {
          q0 = make_double2(0.0, 0.0);
          q1 = make_double2(0.0, 0.0);
        }
        const double aq = aqd[u], v0 = w0[u], v1 = w1[u], v2 = w2[u];
        if (AXIS == 0) {
          // meanfield.py:63-83
          q0 = q0 + cmulri(0.0, -(h * aq - h * v1), e0) - (h * v2) * e1;
          q1 = q1 + cmulri(0.0, -(h * aq + h * v1), e1) + (h * v2) * e0;
          n0 = cmulri(0.0, -h * (aq - v1), a0) - (h * v2) * a1;
          n1 = cmulri(0.0, -h * (aq + v1), a1) + (h * v2) * a0;
        } else if (AXIS == 1) {
          // meanfield.py:92-112
          q0 = q0 + cmulri(0.0, -(h * aq + h * v0), e0) + cmulri(0.0, h * v2, e1);
          q1 = q1 + cmulri(0.0, -(h * aq - h * v0), e1) + cmulri(0.0, h * v2, e0);
          n0 = cmulri(0.0, -h * (aq + v0), a0) + cmulri(0.0, h * v2, a1);
          n1 = cmulri(0.0, -h * (aq - v0), a1) + cmulri(0.0, h * v2, a0);
        } else {
          // meanfield.py:121-141
          q0 = q0 + cmulri(0.0, -(h * aq), e0) + cmulri(h * v0, -(h * v1), e1);
          q1 = q1 + cmulri(0.0, -(h * aq), e1) + cmulri(-(h * v0), -(h * v1), e0);
          n0 = cmulri(0.0, -h * aq, a0) + cmulri(h * v0, -(h * v1), a1);
          n1 = cmulri(0.0, -h * aq, a1) + cmulri(-(h * v0), -(h * v1), a0);
        }
        o[ti][u][0] = q0;
        o[ti][u][1] = q1;
        W[hd_at<N, ROW>(0, line, j)] = n0 - bm[u] * e0;
        W[hd_at<N, ROW>(1, line, j)] = n1 - bm[u] * e1;
      }
    }
  }
  __syncthreads();
  // ---- GEMM 2: r = D w; out = o + r + Nyquist term
#pragma unroll
  for (int ti = 0; ti < G::TMAX; ++ti) {
    const int t = warp + ti * kHdWarps;
    if (t < G::NT) {
      const int j0 = (t / G::LG) * 8, l0 = (t % G::LG) * 8;
      const int j = j0 + (lane >> 2), lp = l0 + 2 * (lane & 3);
      const size_t g0 = gidx(lp, j), g1 = gidx(lp + 1, j);
      const auto pv0 = pre(g0);
      const auto pv1 = pre(g1);
      double acc[4][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
      for (int ks = 0; ks < G::KS; ++ks) {
        const int pt = ks * 4 + (lane & 3);
        const double a = Dm[(j0 + (lane >> 2)) * DLD + pt];
        const double2 x0 = W[hd_at<N, ROW>(0, l0 + (lane >> 2), pt)];
        const double2 x1 = W[hd_at<N, ROW>(1, l0 + (lane >> 2), pt)];
        hd_mma(acc[0], a, x0.x);
        hd_mma(acc[1], a, x0.y);
        hd_mma(acc[2], a, x1.x);
        hd_mma(acc[3], a, x1.y);
      }
      const double nqj = (j & 1) ? -nq : nq;
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int line = lp + u;
        const double sg = nqj * bbar[line];
        const double2 r0 = o[ti][u][0] + make_double2(acc[0][u], acc[1][u]) + sg * alt[line];
        const double2 r1 = o[ti][u][1] + make_double2(acc[2][u], acc[3][u]) + sg * alt[N + line];
        emit(line, j, u == 0 ? g0 : g1, r0, r1, u == 0 ? pv0 : pv1);
      }
    }
  }
  __syncthreads();
}

}  // namespace

namespace {

template <int N>
__device__ __forceinline__ void hd_load_d(double* dst, const double* src) {
  constexpr int DLD = hd_dld<N>();
#pragma unroll 4
  for (int e = threadIdx.x; e < N * N; e += kHdThreads) dst[(e / N) * DLD + e % N] = src[e];
}

// Values an emit step reads from global memory, loaded before its MMAs.
struct HdPre {
  double2 m0, m1;   // the state's partial h psi, both components
  double vp;        // v_pair
};

// A: one x-plane of one state; z lines with the local terms, then y lines.
template <int N>
__global__ void __launch_bounds__(kHdThreads)
hpsi_dmma_x_kernel(const double* __restrict__ pot, const double2* __restrict__ psi, double2* acc, int s0, int nneut,
                   const double* __restrict__ dmat, double nq_y, double nq_z) {
  using G = HdGeo<N>;
  constexpr size_t N2 = (size_t)N * N, N3 = N2 * N;
  constexpr int DLD = hd_dld<N>();
  extern __shared__ __align__(16) unsigned char hd_smem[];
  double2* plane = reinterpret_cast<double2*>(hd_smem);
  double2* wb = plane + G::PLANE;
  double2* alt = wb + G::PLANE;
  double* dz = reinterpret_cast<double*>(alt + 2 * N);
  double* dy = dz + N * DLD;
  double* bbar = dy + N * DLD;
  const int x0 = blockIdx.x, s = s0 + blockIdx.y;
  const double* potq = pot + (size_t)(s >= nneut ? 1 : 0) * 12 * N3;
  const double2* src = psi + (size_t)s * 2 * N3 + (size_t)x0 * N2;
#pragma unroll 6
  for (int e = threadIdx.x; e < 2 * N * N; e += kHdThreads) {
    const int c = e / (N * N), r = e - c * N * N;
    plane[(c * N + r / N) * G::LD + r % N] = src[(size_t)c * N3 + r];
  }
  hd_load_d<N>(dz, dmat + 2 * N2);
  hd_load_d<N>(dy, dmat + 1 * N2);
  __syncthreads();
  double2* dst = acc + (size_t)s * 2 * N3;
  const size_t base = (size_t)x0 * N2;
  hd_pass<N, 2, true, true>(
      plane, wb, dz, alt, bbar, potq, base, N, 1, nq_z, [](size_t) { return 0; },
      [&](int, int, size_t g, double2 q0, double2 q1, int) {
        dst[g] = q0;
        dst[N3 + g] = q1;
      });
  hd_pass<N, 1, false, false>(
      plane, wb, dy, alt, bbar, potq, base, N, 1, nq_y,
      [&](size_t g) { return HdPre{dst[g], dst[N3 + g], 0.0}; },
      [&](int, int, size_t g, double2 q0, double2 q1, const HdPre& pv) {
        dst[g] = pv.m0 + q0;
        dst[N3 + g] = pv.m1 + q1;
      });
}

// B: one y-plane of one state; x lines, then pout = weight * h psi -
// weightuv * v_pair psi, pout_del = v_pair psi and the plane's overlaps.
template <int N>
__global__ void __launch_bounds__(kHdThreads)
hpsi_dmma_y_kernel(const double* __restrict__ pot, const double2* __restrict__ psi, double2* acc, int s0, int nneut,
                   const double* __restrict__ dmat, double nq_x, const double* __restrict__ weight,
                   const double* __restrict__ weightuv, double2* pout, double2* pout_mf, double2* pout_del,
                   double* ovl) {
  using G = HdGeo<N>;
  constexpr size_t N2 = (size_t)N * N, N3 = N2 * N;
  constexpr int DLD = hd_dld<N>();
  extern __shared__ __align__(16) unsigned char hd_smem[];
  __shared__ double red[2][kHdWarps];
  double2* plane = reinterpret_cast<double2*>(hd_smem);
  double2* wb = plane + G::PLANE;
  double2* alt = wb + G::PLANE;
  double* dx = reinterpret_cast<double*>(alt + 2 * N);
  double* bbar = dx + 2 * N * DLD;
  const int y0 = blockIdx.x, s = s0 + blockIdx.y;
  const double* potq = pot + (size_t)(s >= nneut ? 1 : 0) * 12 * N3;
  const double2* src = psi + (size_t)s * 2 * N3 + (size_t)y0 * N;
  // plane (a = x, b = z) at fixed y0
#pragma unroll 6
  for (int e = threadIdx.x; e < 2 * N * N; e += kHdThreads) {
    const int c = e / (N * N), r = e - c * N * N;
    const int a = r / N, b = r % N;
    plane[(c * N + a) * G::LD + b] = src[(size_t)c * N3 + (size_t)a * N2 + b];
  }
  hd_load_d<N>(dx, dmat);
  __syncthreads();
  const double wt = weight ? weight[s] : 1.0;
  const double wu = weightuv ? weightuv[s] : 0.0;
  const double2* a_s = acc + (size_t)s * 2 * N3;
  const size_t so = (size_t)s * 2 * N3;
  double ov_mf = 0.0, ov_po = 0.0;
  hd_pass<N, 0, false, false>(plane, wb, dx, alt, bbar, potq, (size_t)y0 * N, N2, 1, nq_x,
                              [&](size_t g) { return HdPre{a_s[g], a_s[N3 + g], potq[2 * N3 + g]}; },
                              [&](int line, int j, size_t g, double2 q0, double2 q1, const HdPre& pv) {
                                const double vp = pv.vp;
#pragma unroll
                                for (int c = 0; c < 2; ++c) {
                                  const size_t gi = (size_t)c * N3 + g;
                                  const double2 mf = (c == 0 ? pv.m0 : pv.m1) + (c == 0 ? q0 : q1);
                                  const double2 ps = plane[hd_at<N, false>(c, line, j)];
                                  const double2 dl = vp * ps;
                                  const double2 po = wt * mf - wu * dl;
                                  if (pout_mf) pout_mf[so + gi] = mf;
                                  if (pout) pout[so + gi] = po;
                                  if (pout_del) pout_del[so + gi] = dl;
                                  ov_mf += ps.x * mf.x + ps.y * mf.y;
                                  ov_po += ps.x * po.x + ps.y * po.y;
                                }
                              });
  if (ovl) {
    // deterministic block reduction: warp shuffles, then thread 0
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      ov_mf += __shfl_xor_sync(0xffffffffu, ov_mf, o);
      ov_po += __shfl_xor_sync(0xffffffffu, ov_po, o);
    }
    const int w = threadIdx.x / 32, l = threadIdx.x % 32;
    if (l == 0) {
      red[0][w] = ov_mf;
      red[1][w] = ov_po;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double a = 0.0, b = 0.0;
      for (int i = 0; i < kHdWarps; ++i) {
        a += red[0][i];
        b += red[1][i];
      }
      ovl[((size_t)blockIdx.y * N + y0) * 2 + 0] = a;
      ovl[((size_t)blockIdx.y * N + y0) * 2 + 1] = b;
    }
  }
}

template <int N>
int hpsi_dmma_launch_t(hfb_ctx_s* c, const void* pot, int s0, int ns, int nneut, const void* psi,
                       const double* weight, const double* weightuv, void* acc, void* pout, void* pout_mf,
                       void* pout_del, double* ovl, cudaStream_t st) {
  using G = HdGeo<N>;
  if (ns <= 0) return HFB_OK;
  double nq[3];
  for (int a = 0; a < 3; ++a) nq[a] = (M_PI / c->d[a]) * (M_PI / c->d[a]) / N;
  allow_max_dynamic_smem(hpsi_dmma_x_kernel<N>);
  allow_max_dynamic_smem(hpsi_dmma_y_kernel<N>);
  const dim3 grid(N, ns);
  hpsi_dmma_x_kernel<N><<<grid, kHdThreads, G::SMEM, st>>>((const double*)pot, (const double2*)psi, (double2*)acc,
                                                           s0, nneut, c->hpsi_d64, nq[1], nq[2]);
  HFB_CHECK_LAUNCH();
  hpsi_dmma_y_kernel<N><<<grid, kHdThreads, G::SMEM, st>>>((const double*)pot, (const double2*)psi, (double2*)acc,
                                                           s0, nneut, c->hpsi_d64, nq[0], weight, weightuv,
                                                           (double2*)pout, (double2*)pout_mf, (double2*)pout_del,
                                                           ovl);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

}  // namespace

// D of each axis (levels.py:132-189 as a matrix): D[j][l] = -(2 kf / n)
// sum_{k=1}^{n/2-1} k sin(2 pi k (j - l) / n), kf = 2 pi / (n d), in double.
int hpsi_dmma_prepare(hfb_ctx_s* c) {
  c->hpsi_d64 = nullptr;
  const int n = c->n;
  if (n % 8 != 0 || n > 48) return HFB_OK;
  std::vector<double> d((size_t)3 * n * n);
  for (int ax = 0; ax < 3; ++ax) {
    const double kf = 2.0 * M_PI / (n * c->d[ax]);
    for (int j = 0; j < n; ++j)
      for (int l = 0; l < n; ++l) {
        double v = 0.0;
        for (int k = 1; k < n / 2; ++k) {
          const int ph = (((k * (j - l)) % n) + n) % n;
          v += k * sin(2.0 * M_PI * ph / n);
        }
        d[((size_t)ax * n + j) * n + l] = -2.0 * kf / n * v;
      }
  }
  if (cudaMalloc(&c->hpsi_d64, d.size() * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    c->hpsi_d64 = nullptr;
    return HFB_ERR_ALLOC;
  }
  if (cudaMemcpy(c->hpsi_d64, d.data(), d.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
    return HFB_ERR_CUDA;
  return HFB_OK;
}

bool hpsi_dmma_available(hfb_ctx_s* c, int prec) { return prec == HFB_F64 && c->f64_hpsi == 1 && c->hpsi_d64; }

int hpsi_dmma_launch(hfb_ctx_s* c, const void* pot, int s0, int ns, int nneut, const void* psi, const double* weight,
                     const double* weightuv, void* acc, void* pout, void* pout_mf, void* pout_del, double* ovl,
                     cudaStream_t st) {
  return dispatch_n(c->n, [&](auto nn) -> int {
    constexpr int N = decltype(nn)::value;
    return hpsi_dmma_launch_t<N>(c, pot, s0, ns, nneut, psi, weight, weightuv, acc, pout, pout_mf, pout_del, ovl, st);
  });
}

}  // namespace hfb
