// Diagonalisation step: diagstep (static.py:261-461), loewdin_orthonormalize
// (463-482) and construct_hfb_matrices (484-577).
//
//  * Gram contractions C_a = wxyz Psi^H X_a (X = psi, hampsi, hmfpsi,
//    v_pair psi) over K = 2 n^3: one kernel reads each psi tile once for all
//    requested matrices; split-K partials are summed in a fixed order.
//  * Hermitian eigensolver: cyclic two-sided Jacobi in one CTA on the packed
//    lower triangle held in shared memory (round-robin ordering, n/2 disjoint
//    rotations per round); the rotations are recorded and replayed onto the
//    eigenvector matrix by a row-parallel kernel.  Eigenvalues ascending.
//  * small FP64 complex GEMMs for U = S^-1/2 V_lambda, U^H H U, U lambda.
//  * rotation [psi_new | lagrange] = psi [U | U lambda_sym] as one GEMM pass.
#include <math.h>
#include "hfb_ctx.cuh"

namespace hfb {

// ================================================================ Gram ====
// C = wxyz Psi^H X for X in {psi, hampsi, hmfpsi, v_pair psi} (mask bits 0-3)
// over K = 2 n^3.  Work is a list of 48 x 48 output tiles, one matrix per
// tile; S, H and G are Hermitian (Gram matrices of one set of vectors, h
// and v_pair Hermitian) so only tiles with ti <= tj are computed and the
// reduction mirrors them.  Split-K partials are summed in a fixed order.
// 48-state tiles keep the padding of the usual neutron/proton counts small
// (140 -> 144, 96 -> 96); 192 threads (16 x 12) hold 4 x 3 outputs each.
constexpr int GT = 48;        // tile edge (states)
constexpr int GKS = 8;        // k per shared-memory stage
constexpr int GCHUNK = 8192;  // k per split-K chunk (at most; shorter when the grid would be small)
constexpr int GTHREADS = 192;
constexpr int kGramMaxTiles = 160;

struct GramTile {
  unsigned char b, a, ti, tj;   // block (isospin), matrix, tile row, tile column
};
struct GramJob {
  int ntile;
  GramTile t[kGramMaxTiles];
  int s0[2], ns[2];              // state range of each block
  const double* vp[2];           // v_pair for each block (X = v psi)
  int herm_mask;                 // matrices computed on upper tiles only
};

template <class R>
__global__ void __launch_bounds__(GTHREADS)
gram_kernel(GramJob job, size_t K, size_t n3, const cplx<R>* __restrict__ psi, const cplx<R>* __restrict__ hampsi,
            const cplx<R>* __restrict__ hmfpsi, double2* part, int nchunk, int kchunk) {
  using Z = cplx<R>;
  __shared__ Z As[2][GKS][GT + 1];
  __shared__ Z Bs[2][GKS][GT + 1];
  const GramTile tl = job.t[blockIdx.x];
  const int b = tl.b, am = tl.a;
  const int ns = job.ns[b];
  const int i0 = tl.ti * GT, j0 = tl.tj * GT;
  const cplx<R>* P = psi + (size_t)job.s0[b] * K;
  const cplx<R>* X = am == 1 ? hampsi + (size_t)job.s0[b] * K : am == 2 ? hmfpsi + (size_t)job.s0[b] * K : P;
  const double* vp = job.vp[b];
  const size_t k0 = (size_t)blockIdx.y * kchunk;
  const size_t k1 = min(K, k0 + (size_t)kchunk);
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;   // rows ty + 12 u, columns tx + 16 v
  R acc[4][3][2];
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 3; ++v) acc[u][v][0] = acc[u][v][1] = R(0);
  // loader: 48 states x 8 k per operand = 384 elements, two per thread
  auto load = [&](int buf, size_t kb) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int e = threadIdx.x + GTHREADS * h;
      const int st_ = e / GKS, kk = e % GKS;
      const size_t k = kb + kk;
      const bool okk = k < k1;
      const int gi = i0 + st_, gj = j0 + st_;
      As[buf][kk][st_] = (okk && gi < ns) ? P[(size_t)gi * K + k] : czero<Z>();
      Z v = czero<Z>();
      if (okk && gj < ns) {
        v = X[(size_t)gj * K + k];
        if (am == 3) v = (R)vp[k % n3] * v;
      }
      Bs[buf][kk][st_] = v;
    }
  };
  load(0, k0);
  __syncthreads();
  int buf = 0;
  for (size_t kb = k0; kb < k1; kb += GKS) {
    if (kb + GKS < k1) load(buf ^ 1, kb + GKS);
#pragma unroll
    for (int kk = 0; kk < GKS; ++kk) {
      Z av[4], bv[3];
#pragma unroll
      for (int u = 0; u < 4; ++u) av[u] = As[buf][kk][ty + 12 * u];
#pragma unroll
      for (int v = 0; v < 3; ++v) bv[v] = Bs[buf][kk][tx + 16 * v];
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 3; ++v) {
          // conj(a) * b
          acc[u][v][0] += av[u].x * bv[v].x + av[u].y * bv[v].y;
          acc[u][v][1] += av[u].x * bv[v].y - av[u].y * bv[v].x;
        }
    }
    __syncthreads();
    buf ^= 1;
  }
  double2* o = part + ((size_t)blockIdx.x * nchunk + blockIdx.y) * GT * GT;
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 3; ++v)
      o[(ty + 12 * u) * GT + tx + 16 * v] = make_double2((double)acc[u][v][0], (double)acc[u][v][1]);
}

// FP64 states: the same tiles, split-K chunks and partial layout on the
// FP64 tensor cores (mma.sync m8n8k4 .f64).  Over the interleaved storage,
// with k' running over (Re, Im) of each element,
//   Re C_ij = sum_k' a_ik' b_jk',   a = psi_i, b = x_j,
//   Im C_ij = sum_k' a_ik' bt_jk',  bt = (Im x, -Re x) per element,
// so each 8 x 8 output block takes two real MMAs per four k'; bt is b with
// the partner lane's value (one shuffle).  A CTA (4 warps, 24 x 24 outputs
// per warp, 3 x 3 MMA blocks) streams K in stages of GD_KB elements through
// cp.async double buffers (rows padded by one element: the 8 rows a
// fragment load touches fall on distinct bank groups).
constexpr int GD_KB = 16;              // complex k per shared-memory stage
constexpr int GD_LD = GD_KB + 1;       // padded row length (complex)
constexpr int GD_THREADS = 128;
constexpr size_t GD_SMEM = sizeof(double2) * 2 * 2 * GT * GD_LD;

__device__ __forceinline__ void gd_cp16(void* smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((uint32_t)__cvta_generic_to_shared(smem)),
               "l"(gmem)
               : "memory");
}

__device__ __forceinline__ void gd_mma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(GD_THREADS) gram_dmma_kernel(GramJob job, size_t K, size_t n3,
                                                                const double2* __restrict__ psi,
                                                                const double2* __restrict__ hampsi,
                                                                const double2* __restrict__ hmfpsi, double2* part,
                                                                int nchunk, int kchunk) {
  extern __shared__ double2 gd_smem[];
  double2* As = gd_smem;                 // [2][GT][GD_LD]
  double2* Bs = gd_smem + 2 * GT * GD_LD;
  const GramTile tl = job.t[blockIdx.x];
  const int b = tl.b, am = tl.a;
  const int ns = job.ns[b];
  const int i0 = tl.ti * GT, j0 = tl.tj * GT;
  const double2* P = psi + (size_t)job.s0[b] * K;
  const double2* X = am == 1 ? hampsi + (size_t)job.s0[b] * K : am == 2 ? hmfpsi + (size_t)job.s0[b] * K : P;
  const double* vp = job.vp[b];
  const size_t k0 = (size_t)blockIdx.y * kchunk;
  const size_t k1 = min(K, k0 + (size_t)kchunk);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int rw = warp >> 1, cw = warp & 1;
  const int fr = lane >> 2, fk = lane & 3;   // fragment row (A) / column (B), k' within the 4
  double accR[3][3][2], accI[3][3][2];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) accR[i][j][0] = accR[i][j][1] = accI[i][j][0] = accI[i][j][1] = 0.0;
  // one stage: GT rows x GD_KB elements of each operand, consecutive
  // threads on consecutive elements of a row (coalesced)
  auto load = [&](int buf, size_t kb) {
#pragma unroll
    for (int h = 0; h < GT * GD_KB / GD_THREADS; ++h) {
      const int e = threadIdx.x + GD_THREADS * h;
      const int r = e / GD_KB, kk = e % GD_KB;
      const size_t k = kb + kk;
      double2* da = As + ((size_t)buf * GT + r) * GD_LD + kk;
      double2* db = Bs + ((size_t)buf * GT + r) * GD_LD + kk;
      const int gi = i0 + r, gj = j0 + r;
      if (k < k1 && gi < ns) gd_cp16(da, P + (size_t)gi * K + k);
      else *da = make_double2(0.0, 0.0);
      if (k < k1 && gj < ns) {
        if (am == 3) {
          const double2 v = X[(size_t)gj * K + k];
          const double w = vp[k % n3];
          *db = make_double2(w * v.x, w * v.y);
        } else {
          gd_cp16(db, X + (size_t)gj * K + k);
        }
      } else {
        *db = make_double2(0.0, 0.0);
      }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  load(0, k0);
  int buf = 0;
  for (size_t kb = k0; kb < k1; kb += GD_KB) {
    if (kb + GD_KB < k1) {
      load(buf ^ 1, kb + GD_KB);
      asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    }
    __syncthreads();
    const double* A = reinterpret_cast<const double*>(As + (size_t)buf * GT * GD_LD);
    const double* B = reinterpret_cast<const double*>(Bs + (size_t)buf * GT * GD_LD);
#pragma unroll 4
    for (int ks = 0; ks < GD_KB / 2; ++ks) {
      const int kd = 2 * (2 * ks) + fk;      // double index of k' in the row
      double a[3], bv[3], bt[3];
#pragma unroll
      for (int mi = 0; mi < 3; ++mi) a[mi] = A[(24 * rw + 8 * mi + fr) * (2 * GD_LD) + kd];
#pragma unroll
      for (int nj = 0; nj < 3; ++nj) {
        bv[nj] = B[(24 * cw + 8 * nj + fr) * (2 * GD_LD) + kd];
        const double o = __shfl_xor_sync(0xffffffffu, bv[nj], 1);
        bt[nj] = (fk & 1) ? -o : o;
      }
#pragma unroll
      for (int mi = 0; mi < 3; ++mi)
#pragma unroll
        for (int nj = 0; nj < 3; ++nj) {
          gd_mma(accR[mi][nj], a[mi], bv[nj]);
          gd_mma(accI[mi][nj], a[mi], bt[nj]);
        }
    }
    __syncthreads();
    buf ^= 1;
  }
  double2* o = part + ((size_t)blockIdx.x * nchunk + blockIdx.y) * GT * GT;
#pragma unroll
  for (int mi = 0; mi < 3; ++mi)
#pragma unroll
    for (int nj = 0; nj < 3; ++nj)
#pragma unroll
      for (int i = 0; i < 2; ++i)
        o[(24 * rw + 8 * mi + fr) * GT + 24 * cw + 8 * nj + 2 * fk + i] = make_double2(accR[mi][nj][i], accI[mi][nj][i]);
}

struct GramOut {
  double2* p[8];   // [block * 4 + matrix]
};

// out_a[b][i][j] = wxyz * sum over chunks (fixed order); Hermitian matrices
// take the lower triangle from the upper one.
__global__ void gram_reduce_kernel(GramJob job, int nchunk, const double2* part, double scale, GramOut outs,
                                   int ldo) {
  const int t = blockIdx.y;
  const GramTile tl = job.t[t];
  const int b = tl.b, am = tl.a;
  const int ns = job.ns[b];
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= GT * GT) return;
  const int li = e / GT, lj = e % GT;
  const int i = tl.ti * GT + li, j = tl.tj * GT + lj;
  if (i >= ns || j >= ns) return;
  double re = 0, im = 0;
  const double2* p = part + (size_t)t * nchunk * GT * GT + e;
  for (int c = 0; c < nchunk; ++c) {
    const double2 v = p[(size_t)c * GT * GT];
    re += v.x;
    im += v.y;
  }
  double2* out = outs.p[b * 4 + am];
  const bool herm = (job.herm_mask >> am) & 1;
  if (herm && i > j) return;           // written from the mirrored element below
  out[(size_t)i * ldo + j] = make_double2(scale * re, scale * im);
  if (herm && i != j) out[(size_t)j * ldo + i] = make_double2(scale * re, -scale * im);
}

int gram_tc_launch(hfb_ctx_s* c, int nblk, const int* s0, const int* ns, const int* masks, const void* psi,
                   const void* hampsi, const void* hmfpsi, const double* const* vp, double wxyz,
                   double2* const* outs_host, int ldo, cudaStream_t st);   // gram_tc.cu

// One launch for the requested matrices of up to two state blocks.
// outs[b * 4 + a] receives matrix a of block b (leading dimension ldo).

int gram_launch(hfb_ctx_s* c, int prec, int nblk, const int* s0, const int* ns, const int* masks, const void* psi,
                const void* hampsi, const void* hmfpsi, const double* const* vp, double wxyz, double2* const* outs_host,
                int ldo, cudaStream_t st) {
  // single precision: tensor cores (three-term tf32) unless disabled for this context
  if (prec != HFB_F64 && c->use_tcgen05) {
    const int r = gram_tc_launch(c, nblk, s0, ns, masks, psi, hampsi, hmfpsi, vp, wxyz, outs_host, ldo, st);
    if (r != HFB_ERR_UNSUPPORTED_GRID) return r;
  }
  const size_t n3 = (size_t)c->n * c->n * c->n, K = 2 * n3;
  int kchunk = GCHUNK;   // set below from the tile count
  GramJob job{};
  job.herm_mask = 1 | 4 | 8;
  for (int b = 0; b < nblk; ++b) {
    job.s0[b] = s0[b];
    job.ns[b] = ns[b];
    job.vp[b] = vp ? vp[b] : nullptr;
    const int nt = (ns[b] + GT - 1) / GT;
    for (int a = 0; a < 4; ++a) {
      if (!(masks[b] & (1 << a)) || ns[b] <= 0) continue;
      const bool herm = (job.herm_mask >> a) & 1;
      for (int ti = 0; ti < nt; ++ti)
        for (int tj = herm ? ti : 0; tj < nt; ++tj) {
          if (job.ntile >= kGramMaxTiles) return HFB_ERR_ARG;
          job.t[job.ntile++] = GramTile{(unsigned char)b, (unsigned char)a, (unsigned char)ti, (unsigned char)tj};
        }
    }
  }
  if (job.ntile == 0) return HFB_OK;
  // split K so that the grid has about two CTAs per SM even for few tiles
  // and short K (small grids): chunks a multiple of 64 elements, at most
  // GCHUNK
  {
    const size_t want = (size_t)(2 * 148 + job.ntile - 1) / job.ntile;
    size_t kc = (K + want - 1) / want;
    kc = (kc + 63) / 64 * 64;
    if (kc < 256) kc = 256;
    if (kc > (size_t)GCHUNK) kc = GCHUNK;
    kchunk = (int)kc;
  }
  const int nchunk = (int)((K + kchunk - 1) / kchunk);
  double2* part = (double2*)scratch(c, hfb_ctx_s::S_GRAM, sizeof(double2) * (size_t)job.ntile * nchunk * GT * GT);
  if (!part) return HFB_ERR_ALLOC;
  GramOut ot;
  for (int q = 0; q < 8; ++q) ot.p[q] = outs_host[q];
  dim3 grid(job.ntile, nchunk);
  if (prec == HFB_F64 && c->f64_mma) {
    static const bool smem_ok =
        cudaFuncSetAttribute(gram_dmma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GD_SMEM) ==
        cudaSuccess;
    if (!smem_ok) return HFB_ERR_CUDA;
    gram_dmma_kernel<<<grid, GD_THREADS, GD_SMEM, st>>>(job, K, n3, (const double2*)psi, (const double2*)hampsi,
                                                     (const double2*)hmfpsi, part, nchunk, kchunk);
  } else if (prec == HFB_F64)
    gram_kernel<double><<<grid, GTHREADS, 0, st>>>(job, K, n3, (const double2*)psi, (const double2*)hampsi,
                                              (const double2*)hmfpsi, part, nchunk, kchunk);
  else
    gram_kernel<float><<<grid, GTHREADS, 0, st>>>(job, K, n3, (const float2*)psi, (const float2*)hampsi,
                                             (const float2*)hmfpsi, part, nchunk, kchunk);
  HFB_CHECK_LAUNCH();
  dim3 g2((GT * GT + 255) / 256, job.ntile);
  gram_reduce_kernel<<<g2, 256, 0, st>>>(job, nchunk, part, wxyz, ot, ldo);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

// ============================================================== Jacobi ====
// Packed lower triangle: element (k, l), k >= l, at k (k + 1) / 2 + l.
__device__ __forceinline__ int pk(int k, int l) { return k * (k + 1) / 2 + l; }
__device__ __forceinline__ double2 ld_h(const double2* a, int k, int l) {
  if (k >= l) return a[pk(k, l)];
  double2 v = a[pk(l, k)];
  return make_double2(v.x, -v.y);
}
__device__ __forceinline__ void st_h(double2* a, int k, int l, double2 v) {
  if (k >= l) a[pk(k, l)] = v;
  else a[pk(l, k)] = make_double2(v.x, -v.y);
}

// Round-robin tournament: round r of m-1 (m even), pair index q < m/2.
__device__ __forceinline__ void rr_pair(int m, int r, int q, int& a, int& b) {
  if (q == 0) { a = r % (m - 1); b = m - 1; }
  else { a = (r + q) % (m - 1); b = (r + m - 1 - q) % (m - 1); }
  if (a > b) { int t = a; a = b; b = t; }
}

struct Pair2 {
  int v[2];
};

struct JacRot {
  double cs, sn;
  double2 om;   // exp(-i phi)
};

constexpr int kJacMaxSweeps = 40;
constexpr int kEighMax = 4;     // matrices per batched launch
constexpr int kJacThreads = 1024;
constexpr int kJacBlk = 4;      // 2x2 blocks per thread (half*(half+1)/2 <= 4096 -> n <= 180)

// One batched solve: up to kEighMax independent matrices, one CTA each.
struct EighBatch {
  int nb;
  int n[kEighMax];
  int lda[kEighMax];
  const double2* a[kEighMax];
  double* w[kEighMax];
  double2* v[kEighMax];
  int vblk0[kEighMax + 1];     // prefix of row blocks for the vector replay
  int* sweeps;                 // optional device output [nb]: sweeps used
  double tol_rel;              // off-diagonal threshold relative to ||A||_F (0: double eps)
  int stage_half;              // rotations per round in the replay's staging buffer (set by eigh_batch)
  const int* gate;             // optional device flag: the solve runs only when *gate != 0
};

// One CTA per matrix: cyclic two-sided Jacobi on the packed lower triangle.
// Each round applies n/2 disjoint rotations (round-robin pairing); thread t
// owns fixed 2x2 blocks (pair q1 rows x pair q2 columns, q1 >= q2) for the
// whole solve, and skips a block when both of its rotations are the
// identity.  Rotations are recorded for the eigenvector replay.
__global__ void __launch_bounds__(kJacThreads)
jacobi_kernel(EighBatch eb, JacRot* rot, int* nrounds_out, int* status, size_t rot_stride) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (eb.gate && *eb.gate == 0) return;
  const int b = blockIdx.x;
  const int n = eb.n[b], lda = eb.lda[b];
  const int m = n + (n & 1);   // pad odd sizes with a decoupled index
  const int half = m / 2;
  double2* a = reinterpret_cast<double2*>(smem_raw);
  JacRot* rr = reinterpret_cast<JacRot*>(a + (size_t)m * (m + 1) / 2);
  int* rp = reinterpret_cast<int*>(rr + half);
  int* rq = rp + half;
  int* act = rq + half;
  __shared__ int any_rot;
  __shared__ int round_rot[2];   // a rotation in round r (parity r & 1)
  const double2* Ab = eb.a[b];
  JacRot* rotb = rot + (size_t)b * rot_stride;
  // the lower triangle (eigh with symmetrize_input=False reads only it; the
  // diagonal's imaginary part is ignored as by LAPACK heevd)
  for (int e = threadIdx.x; e < m * (m + 1) / 2; e += blockDim.x) {
    int k = (int)((sqrt(8.0 * e + 1.0) - 1.0) / 2.0);
    while (k * (k + 1) / 2 > e) --k;
    while ((k + 1) * (k + 2) / 2 <= e) ++k;
    const int l = e - k * (k + 1) / 2;
    double2 v = make_double2(0.0, 0.0);
    if (k < n && l < n) v = Ab[(size_t)k * lda + l];
    if (k == l) v.y = 0.0;
    a[e] = v;
  }
  // Frobenius norm (invariant under the rotations): an off-diagonal element
  // below eps ||A||_F is at the rounding-noise level the rotations
  // themselves create, so it is not rotated (the eigenvalue error this
  // leaves is second order in it)
  __shared__ double red_f[32];
  __shared__ double tol_abs;
  {
    double f2 = 0.0;
    for (int e = threadIdx.x; e < m * (m + 1) / 2; e += blockDim.x) {
      int k = (int)((sqrt(8.0 * e + 1.0) - 1.0) / 2.0);
      while (k * (k + 1) / 2 > e) --k;
      while ((k + 1) * (k + 2) / 2 <= e) ++k;
      const int l = e - k * (k + 1) / 2;
      double v = 0.0;
      if (k < n && l < n) {
        const double2 x = Ab[(size_t)k * lda + l];
        v = (k == l ? x.x * x.x : 2.0 * (x.x * x.x + x.y * x.y));
      }
      f2 += v;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) f2 += __shfl_xor_sync(0xffffffffu, f2, o);
    if ((threadIdx.x & 31) == 0) red_f[threadIdx.x / 32] = f2;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < (int)(blockDim.x / 32); ++w) t += red_f[w];
      tol_abs = (eb.tol_rel > 0.0 ? eb.tol_rel : 2.220446049250313e-16) * sqrt(t);
    }
  }
  // this thread's blocks (round independent)
  const int nblk = half * (half + 1) / 2;
  int bq1[kJacBlk], bq2[kJacBlk];
#pragma unroll
  for (int j = 0; j < kJacBlk; ++j) {
    const int e = threadIdx.x + j * kJacThreads;
    bq1[j] = bq2[j] = -1;
    if (e < nblk) {
      int q1 = (int)((sqrt(8.0 * e + 1.0) - 1.0) / 2.0);
      while (q1 * (q1 + 1) / 2 > e) --q1;
      while ((q1 + 1) * (q1 + 2) / 2 <= e) ++q1;
      bq1[j] = q1;
      bq2[j] = e - q1 * (q1 + 1) / 2;
    }
  }
  __syncthreads();
  int rounds = 0;
  int sweep = 0;
  for (; sweep < kJacMaxSweeps; ++sweep) {
    if (threadIdx.x == 0) any_rot = 0;
    __syncthreads();
    // a sweep in which every pair is negligible at its start rotates nothing
    // (the matrix never changes), so it is skipped after one parallel check
    // of all pairs instead of being run round by round
    {
      int need = 0;
      for (int e = threadIdx.x; e < m * (m - 1) / 2 && !need; e += blockDim.x) {
        int k = (int)((sqrt(8.0 * e + 1.0) - 1.0) / 2.0);
        while (k * (k + 1) / 2 > e) --k;
        while ((k + 1) * (k + 2) / 2 <= e) ++k;
        const int p_ = k + 1, q_ = e - k * (k + 1) / 2;   // p_ > q_
        const double app = a[pk(p_, p_)].x, aqq = a[pk(q_, q_)].x;
        const double2 apq = ld_h(a, p_, q_);
        const double mag = hypot(apq.x, apq.y);
        const bool negl = (mag <= tol_abs) ||
                          (fabs(app) + 100.0 * mag == fabs(app) && fabs(aqq) + 100.0 * mag == fabs(aqq));
        if (!negl) need = 1;
      }
      if (need) any_rot = 1;
      __syncthreads();
      const int go = any_rot;
      __syncthreads();
      if (!go) break;
      if (threadIdx.x == 0) any_rot = 0;
      __syncthreads();
    }
    if (threadIdx.x == 0) round_rot[0] = round_rot[1] = 0;
    __syncthreads();
    for (int r = 0; r < m - 1; ++r) {
      // the next round's flag is cleared here; no thread reads it before
      // this round's barrier
      if (threadIdx.x == 0) round_rot[(r + 1) & 1] = 0;
      for (int q = threadIdx.x; q < half; q += blockDim.x) {
        int p_, q_;
        rr_pair(m, r, q, p_, q_);
        JacRot g;
        g.cs = 1.0; g.sn = 0.0; g.om = make_double2(1.0, 0.0);
        const double app = a[pk(p_, p_)].x, aqq = a[pk(q_, q_)].x;
        const double2 apq = ld_h(a, p_, q_);
        const double mag = hypot(apq.x, apq.y);
        // negligible off-diagonal element relative to both diagonal entries
        const bool negl = (mag <= tol_abs) ||
                          (fabs(app) + 100.0 * mag == fabs(app) && fabs(aqq) + 100.0 * mag == fabs(aqq));
        int on = 0;
        if (!negl) {
          const double theta = (aqq - app) / (2.0 * mag);
          double t = 1.0 / (fabs(theta) + sqrt(theta * theta + 1.0));
          if (theta < 0.0) t = -t;
          g.cs = 1.0 / sqrt(t * t + 1.0);
          g.sn = t * g.cs;
          g.om = make_double2(apq.x / mag, -apq.y / mag);
          on = 1;
          any_rot = 1;
          round_rot[r & 1] = 1;
        }
        rr[q] = g;
        rp[q] = p_;
        rq[q] = q_;
        act[q] = on;
        rotb[(size_t)rounds * half + q] = g;
      }
      __syncthreads();
      // a round without rotations leaves the matrix as it is: no update
      // pass and no second barrier (the next round's first writes to the
      // rotation arrays come after every thread has passed this test)
      if (!round_rot[r & 1]) {
        ++rounds;
        continue;
      }
#pragma unroll
      for (int j = 0; j < kJacBlk; ++j) {
        const int q1 = bq1[j], q2 = bq2[j];
        if (q1 < 0) continue;
        const int a1 = act[q1], a2 = act[q2];
        if (!a1 && !a2) continue;
        const int k0 = rp[q1], k1 = rq[q1];
        const JacRot g1 = rr[q1];
        if (q1 == q2) {
          const double app = a[pk(k0, k0)].x, aqq = a[pk(k1, k1)].x;
          const double2 apq = ld_h(a, k0, k1);
          const double mag = hypot(apq.x, apq.y);
          const double t = g1.sn / g1.cs;
          a[pk(k0, k0)] = make_double2(app - t * mag, 0.0);
          a[pk(k1, k1)] = make_double2(aqq + t * mag, 0.0);
          st_h(a, k1, k0, make_double2(0.0, 0.0));
          continue;
        }
        const int l0 = rp[q2], l1 = rq[q2];
        const JacRot g2 = rr[q2];
        // G = [[cs, sn], [-sn om, cs om]] (rows: old index, cols: new index)
        double2 B00 = ld_h(a, k0, l0), B01 = ld_h(a, k0, l1), B10 = ld_h(a, k1, l0), B11 = ld_h(a, k1, l1);
        auto cm = [](double2 x, double2 y) { return make_double2(x.x * y.x - x.y * y.y, x.x * y.y + x.y * y.x); };
        if (a2) {   // right multiply by G2 (columns l0, l1)
          const double2 t10 = cm(B01, g2.om), t11 = cm(B11, g2.om);
          const double2 c00 = make_double2(g2.cs * B00.x - g2.sn * t10.x, g2.cs * B00.y - g2.sn * t10.y);
          const double2 c01 = make_double2(g2.sn * B00.x + g2.cs * t10.x, g2.sn * B00.y + g2.cs * t10.y);
          const double2 c10 = make_double2(g2.cs * B10.x - g2.sn * t11.x, g2.cs * B10.y - g2.sn * t11.y);
          const double2 c11 = make_double2(g2.sn * B10.x + g2.cs * t11.x, g2.sn * B10.y + g2.cs * t11.y);
          B00 = c00; B01 = c01; B10 = c10; B11 = c11;
        }
        if (a1) {   // left multiply by G1^H = [[cs, -sn conj(om)], [sn, cs conj(om)]] (rows k0, k1)
          const double2 oc = make_double2(g1.om.x, -g1.om.y);
          const double2 u0 = cm(B10, oc), u1 = cm(B11, oc);
          const double2 d00 = make_double2(g1.cs * B00.x - g1.sn * u0.x, g1.cs * B00.y - g1.sn * u0.y);
          const double2 d01 = make_double2(g1.cs * B01.x - g1.sn * u1.x, g1.cs * B01.y - g1.sn * u1.y);
          const double2 d10 = make_double2(g1.sn * B00.x + g1.cs * u0.x, g1.sn * B00.y + g1.cs * u0.y);
          const double2 d11 = make_double2(g1.sn * B01.x + g1.cs * u1.x, g1.sn * B01.y + g1.cs * u1.y);
          B00 = d00; B01 = d01; B10 = d10; B11 = d11;
        }
        st_h(a, k0, l0, B00);
        st_h(a, k0, l1, B01);
        st_h(a, k1, l0, B10);
        st_h(a, k1, l1, B11);
      }
      __syncthreads();
      ++rounds;
    }
    const int cont = any_rot;
    __syncthreads();
    if (!cont) break;
  }
  if (threadIdx.x == 0) {
    nrounds_out[b] = rounds;
    if (eb.sweeps) eb.sweeps[b] = sweep + 1;
    if (sweep >= kJacMaxSweeps) latch_error(status, HFB_ERR_NO_CONVERGENCE);
  }
  double* wb = eb.w[b];
  for (int k = threadIdx.x; k < n; k += blockDim.x) wb[k] = a[pk(k, k)].x;
}

// Replay V = I G_1 G_2 ... onto blocks of kVecRows rows, then order the
// columns by ascending eigenvalue (stable for ties).  The recorded rotations
// are streamed through shared memory kVecChunk rounds at a time with
// cp.async double buffering, so each round costs one block barrier instead
// of one global-memory latency.
constexpr int kVecRows = 8;
constexpr int kVecChunk = 8;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

__global__ void __launch_bounds__(256)
jacobi_vectors_kernel(EighBatch eb, const JacRot* __restrict__ rot, const int* __restrict__ nrounds,
                      size_t rot_stride) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (eb.gate && *eb.gate == 0) return;
  int b = 0;
  while (b + 1 < eb.nb && (int)blockIdx.x >= eb.vblk0[b + 1]) ++b;
  const int rb = blockIdx.x - eb.vblk0[b];
  const int n = eb.n[b], lda = eb.lda[b];
  const int m = n + (n & 1), half = m / 2;
  JacRot* stage = reinterpret_cast<JacRot*>(smem_raw);                      // [2][kVecChunk][hmax]
  const int hmax = eb.stage_half;
  double2* v = reinterpret_cast<double2*>(stage + 2 * kVecChunk * hmax);    // [kVecRows][m]
  int* order = reinterpret_cast<int*>(v + (size_t)kVecRows * m);
  const int r0 = rb * kVecRows;
  for (int e = threadIdx.x; e < kVecRows * m; e += blockDim.x) {
    const int i = e / m, j = e % m;
    v[e] = make_double2((r0 + i) == j ? 1.0 : 0.0, 0.0);
  }
  const JacRot* rb_ = rot + (size_t)b * rot_stride;
  const int nr = nrounds[b];
  const int nchunk = (nr + kVecChunk - 1) / kVecChunk;
  auto stage_load = [&](int c) {
    if (c < nchunk) {
      const int rs = c * kVecChunk;
      const int cnt = (nr - rs < kVecChunk ? nr - rs : kVecChunk) * half;   // rotations in this chunk
      const char* src = reinterpret_cast<const char*>(rb_ + (size_t)rs * half);
      char* dst = reinterpret_cast<char*>(stage + (size_t)(c & 1) * kVecChunk * hmax);
      for (int e = threadIdx.x; e < 2 * cnt; e += blockDim.x) cp_async16(dst + 16 * e, src + 16 * e);
    }
    cp_async_commit();
  };
  stage_load(0);
  for (int c = 0; c < nchunk; ++c) {
    stage_load(c + 1);
    cp_async_wait1();
    __syncthreads();
    const JacRot* sg = stage + (size_t)(c & 1) * kVecChunk * hmax;
    const int rs = c * kVecChunk;
    const int re = nr - rs < kVecChunk ? nr : rs + kVecChunk;
    for (int r = rs; r < re; ++r) {
      const int rr_ = r % (m - 1);
      const JacRot* gr = sg + (size_t)(r - rs) * half;
      for (int e = threadIdx.x; e < kVecRows * half; e += blockDim.x) {
        const int i = e / half, q = e % half;
        const JacRot g = gr[q];
        if (g.sn == 0.0) continue;
        int p_, q_;
        rr_pair(m, rr_, q, p_, q_);
        const double2 vp = v[i * m + p_], vq = v[i * m + q_];
        const double2 t = make_double2(vq.x * g.om.x - vq.y * g.om.y, vq.x * g.om.y + vq.y * g.om.x);
        v[i * m + p_] = make_double2(g.cs * vp.x - g.sn * t.x, g.cs * vp.y - g.sn * t.y);
        v[i * m + q_] = make_double2(g.sn * vp.x + g.cs * t.x, g.sn * vp.y + g.cs * t.y);
      }
      __syncthreads();
    }
  }
  const double* wb = eb.w[b];
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    int rank = 0;
    const double wj = wb[j];
    for (int k = 0; k < n; ++k) {
      const double wk = wb[k];
      rank += (wk < wj) || (wk == wj && k < j);
    }
    order[rank] = j;
  }
  __syncthreads();
  double2* Vb = eb.v[b];
  for (int e = threadIdx.x; e < kVecRows * n; e += blockDim.x) {
    const int i = e / n, c = e % n;
    if (r0 + i < n) Vb[(size_t)(r0 + i) * lda + c] = v[i * m + order[c]];
  }
}

__global__ void sort_values_kernel(EighBatch eb) {
  if (eb.gate && *eb.gate == 0) return;
  const int b = blockIdx.x;
  const int n = eb.n[b];
  extern __shared__ double tmpw[];
  double* wb = eb.w[b];
  for (int j = threadIdx.x; j < n; j += blockDim.x) tmpw[j] = wb[j];
  __syncthreads();
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    int rank = 0;
    const double wj = tmpw[j];
    for (int k = 0; k < n; ++k) rank += (tmpw[k] < wj) || (tmpw[k] == wj && k < j);
    wb[rank] = wj;
  }
}

// Batched Hermitian eigensolver over the matrices of ``eb`` (all concurrent).
int eigh_batch(hfb_ctx_s* c, EighBatch eb, cudaStream_t st) {
  if (eb.nb <= 0) return HFB_OK;
  int mmax = 0, nmax = 0;
  eb.vblk0[0] = 0;
  for (int i = 0; i < eb.nb; ++i) {
    if (eb.n[i] <= 0 || eb.lda[i] < eb.n[i]) return HFB_ERR_ARG;
    const int m = eb.n[i] + (eb.n[i] & 1);
    mmax = m > mmax ? m : mmax;
    nmax = eb.n[i] > nmax ? eb.n[i] : nmax;
    eb.vblk0[i + 1] = eb.vblk0[i] + (eb.n[i] + kVecRows - 1) / kVecRows;
  }
  const int half = mmax / 2;
  if (half * (half + 1) / 2 > kJacBlk * kJacThreads) return HFB_ERR_ARG;
  const size_t smem = sizeof(double2) * (size_t)mmax * (mmax + 1) / 2 + (sizeof(JacRot) + 3 * sizeof(int)) * half;
  if (smem > 227 * 1024) return HFB_ERR_ARG;
  const size_t rot_stride = (size_t)kJacMaxSweeps * (mmax - 1) * half;
  char* buf = (char*)scratch(c, hfb_ctx_s::S_MAT, sizeof(JacRot) * rot_stride * eb.nb + sizeof(int) * kEighMax + 64);
  if (!buf) return HFB_ERR_ALLOC;
  JacRot* rot = (JacRot*)buf;
  int* nr = (int*)(buf + sizeof(JacRot) * rot_stride * eb.nb);
  allow_max_dynamic_smem(jacobi_kernel);
  jacobi_kernel<<<eb.nb, kJacThreads, smem, st>>>(eb, rot, nr, c->dev_status, rot_stride);
  HFB_CHECK_LAUNCH();
  eb.stage_half = half;
  const size_t smem2 =
      sizeof(JacRot) * 2 * kVecChunk * half + sizeof(double2) * kVecRows * mmax + sizeof(int) * mmax;
  allow_max_dynamic_smem(jacobi_vectors_kernel);
  jacobi_vectors_kernel<<<eb.vblk0[eb.nb], 256, smem2, st>>>(eb, rot, nr, rot_stride);
  HFB_CHECK_LAUNCH();
  sort_values_kernel<<<eb.nb, 256, sizeof(double) * nmax, st>>>(eb);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

// nb matrices a[nb][n][lda] -> w[nb][n] ascending, v[nb][n][lda].
int eigh_launch(hfb_ctx_s* c, int nb, int n, int lda, const double2* a, double* w, double2* v, int* sweeps,
                cudaStream_t st) {
  for (int b0 = 0; b0 < nb; b0 += kEighMax) {
    EighBatch eb{};
    eb.sweeps = sweeps ? sweeps + b0 : nullptr;
    eb.nb = nb - b0 < kEighMax ? nb - b0 : kEighMax;
    for (int i = 0; i < eb.nb; ++i) {
      eb.n[i] = n;
      eb.lda[i] = lda;
      eb.a[i] = a + (size_t)(b0 + i) * n * lda;
      eb.w[i] = w + (size_t)(b0 + i) * n;
      eb.v[i] = v + (size_t)(b0 + i) * n * lda;
    }
    int r = eigh_batch(c, eb, st);
    if (r) return r;
  }
  return HFB_OK;
}

// ========================================================= small GEMMs ====
// C[b] = alpha A'[b] B'[b] + dadd I with A' = A or A^H, B' = B or B^H;
// n x n, leading dim ld, batched over blockIdx.z with per-batch strides.
// When ``gate`` is given the kernel does nothing if gate_k > *gate (used to
// retire converged Newton-Schulz steps without a host round trip).
__global__ void zgemm_small_kernel(int n, int ld, int ta, int tb, const double2* A, size_t sa, const double2* B,
                                   size_t sb, double2* C, size_t sc, Pair2 nper, double alpha, double dadd,
                                   const int* gate, int gate_k) {
  __shared__ double2 As[16][17], Bs[16][17];
  if (gate && gate_k > *gate) return;
  const int b = blockIdx.z;
  const int nb = nper.v[b] > 0 ? nper.v[b] : n;
  const int i = blockIdx.y * 16 + threadIdx.y, j = blockIdx.x * 16 + threadIdx.x;
  if (blockIdx.y * 16 >= nb || blockIdx.x * 16 >= nb) return;
  const double2* Ab = A + b * sa;
  const double2* Bb = B + b * sb;
  double re = 0, im = 0;
  for (int k0 = 0; k0 < nb; k0 += 16) {
    const int ka = k0 + threadIdx.x, kb = k0 + threadIdx.y;
    double2 av = make_double2(0, 0), bv = make_double2(0, 0);
    if (i < nb && ka < nb) {
      if (ta) { av = Ab[(size_t)ka * ld + i]; av.y = -av.y; }
      else av = Ab[(size_t)i * ld + ka];
    }
    if (j < nb && kb < nb) {
      if (tb) { bv = Bb[(size_t)j * ld + kb]; bv.y = -bv.y; }
      else bv = Bb[(size_t)kb * ld + j];
    }
    As[threadIdx.y][threadIdx.x] = av;
    Bs[threadIdx.y][threadIdx.x] = bv;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const double2 x = As[threadIdx.y][k], y = Bs[k][threadIdx.x];
      re += x.x * y.x - x.y * y.y;
      im += x.x * y.y + x.y * y.x;
    }
    __syncthreads();
  }
  if (i < nb && j < nb)
    C[b * sc + (size_t)i * ld + j] = make_double2(alpha * re + (i == j ? dadd : 0.0), alpha * im);
}

static int zgemm_small(int nmax, int ld, int ta, int tb, const double2* A, size_t sa, const double2* B, size_t sb,
                       double2* C, size_t sc, Pair2 nper, int batch, cudaStream_t st, double alpha = 1.0,
                       double dadd = 0.0, const int* gate = nullptr, int gate_k = 0) {
  dim3 grid((nmax + 15) / 16, (nmax + 15) / 16, batch);
  zgemm_small_kernel<<<grid, dim3(16, 16), 0, st>>>(nmax, ld, ta, tb, A, sa, B, sb, C, sc, nper, alpha, dadd, gate,
                                                    gate_k);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

// One n x n product C = A' B' (A' = A or A^H, B' = B or B^H), leading
// dimension ld, for other translation units.
int zgemm_small_one(int n, int ld, int ta, int tb, const double2* A, const double2* B, double2* C, cudaStream_t st) {
  Pair2 nper;
  nper.v[0] = n;
  nper.v[1] = 0;
  return zgemm_small(n, ld, ta, tb, A, 0, B, 0, C, 0, nper, 1, st);
}

// ------------------------------------------ Hermitian eigen refinement ----
// Eigenpairs of a Hermitian matrix that is already nearly diagonal in the
// current basis (lambda after a gradient step: the states are the previous
// eigenvectors), by the iterative refinement of Ogita and Aishima (Japan J.
// Indust. Appl. Math. 35, 2018; clustered eigenvalues: 36, 2019).  From X
// (start I):
//   R = I - X^H X,  S = X^H A X,  l_i = Re S_ii / (1 - Re R_ii),
//   d = 2 (||S - diag(l)||_F + ||A||_F ||R||_F),
//   E_ij = (S_ij + l_j R_ij) / (l_j - l_i)  if |l_i - l_j| > d,  R_ij / 2 else,
//   X <- X (I + E),
// quadratically convergent for the pairs separated by more than d.  The
// pairs the last step left coupled (Kramers pairs, accidental
// near-degeneracies) form clusters that are diagonalised exactly as small
// blocks of the final X^H A X; the eigenpairs are sorted ascending and
// accepted only if V^H A V is diagonal and V^H V = I to the requested
// accuracy.  Only GEMMs on many SMs and a few small kernels: no single-CTA
// sweep.  When the refinement has not converged after kRefMaxIt steps, a
// cluster has more than kClusterMax members or the acceptance test fails,
// the Jacobi solver runs instead (its kernels are gated on a device flag, so
// the choice needs no host round trip).
constexpr int kRefMaxIt = 6;
constexpr int kClusterMax = 16;   // a j = 15/2 shell of a near-spherical nucleus
constexpr int kRefMaxN = 256;

struct RefWork {
  double2 *Ah, *X0, *X1, *AX, *S, *R, *E, *Xf, *Q;   // [nb][ld][ld] each; Q [nb][ld][kClusterMax]
  double *lam, *ev, *anorm, *dlt;                    // [nb][ld], [nb][ld], [nb], [nb]
  int *conv, *rdone, *fallback, *cinfo;              // conv [nb], cinfo [nb][ld][4]
};

__device__ __forceinline__ double block_sum(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x / 32] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < (int)(blockDim.x / 32); ++w) t += red[w];
  return t;
}

// Ah = the Hermitian matrix of the lower triangle of A (the diagonal's
// imaginary part dropped, as eigh with UPLO='L'), X0 = I, ||Ah||_F; flags reset.
__global__ void ref_init_kernel(int ld, Pair2 nper, const double2* A, size_t sA, RefWork w) {
  __shared__ double red[32];
  const int b = blockIdx.x, n = nper.v[b];
  const size_t sm = (size_t)ld * ld;
  const double2* Ab = A + b * sA;
  double f2 = 0.0;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int i = e / n, j = e % n;
    double2 v = i >= j ? Ab[(size_t)i * ld + j] : Ab[(size_t)j * ld + i];
    if (i < j) v.y = -v.y;
    if (i == j) v.y = 0.0;
    w.Ah[b * sm + (size_t)i * ld + j] = v;
    w.X0[b * sm + (size_t)i * ld + j] = make_double2(i == j ? 1.0 : 0.0, 0.0);
    f2 += v.x * v.x + v.y * v.y;
  }
  const double t = block_sum(f2, red);
  if (threadIdx.x == 0) {
    w.anorm[b] = sqrt(t);
    w.conv[b] = 0;
    if (b == 0) {
      *w.rdone = 1 << 30;
      *w.fallback = 0;
    }
  }
}

// One refinement step for matrix b: l, d, E' = I + E; conv[b] when the
// coupling of the separated pairs and the loss of orthonormality are small.
__global__ void ref_update_kernel(int ld, Pair2 nper, RefWork w, int k, double tol) {
  __shared__ double red[32];
  __shared__ double lam[kRefMaxN];
  if (k > *w.rdone) return;
  const int b = blockIdx.x, n = nper.v[b];
  const size_t sm = (size_t)ld * ld;
  const double2* S = w.S + b * sm;
  const double2* R = w.R + b * sm;
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    lam[i] = S[(size_t)i * ld + i].x / (1.0 - R[(size_t)i * ld + i].x);
  __syncthreads();
  double o2 = 0.0, r2 = 0.0;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int i = e / n, j = e % n;
    const double2 sv = S[(size_t)i * ld + j], rv = R[(size_t)i * ld + j];
    const double dx = i == j ? sv.x - lam[i] : sv.x;
    o2 += dx * dx + sv.y * sv.y;
    r2 += rv.x * rv.x + rv.y * rv.y;
  }
  const double off = sqrt(block_sum(o2, red)), rn = sqrt(block_sum(r2, red));
  const double an = w.anorm[b];
  const double d = 2.0 * (off + an * rn);
  double nc2 = 0.0;
  double2* E = w.E + b * sm;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int i = e / n, j = e % n;
    const double2 sv = S[(size_t)i * ld + j], rv = R[(size_t)i * ld + j];
    double2 ev;
    if (i == j) {
      ev = make_double2(1.0 + 0.5 * rv.x, 0.5 * rv.y);
    } else if (fabs(lam[i] - lam[j]) > d) {
      const double den = lam[j] - lam[i];
      ev = make_double2((sv.x + lam[j] * rv.x) / den, (sv.y + lam[j] * rv.y) / den);
      nc2 += sv.x * sv.x + sv.y * sv.y;
    } else {
      ev = make_double2(0.5 * rv.x, 0.5 * rv.y);
    }
    E[(size_t)i * ld + j] = ev;
  }
  const double nc = sqrt(block_sum(nc2, red));
  if (threadIdx.x == 0) {
    w.dlt[b] = d;
    // ||I - X^H X||_F cannot go below the rounding of the n-term sums
    w.conv[b] = (nc <= tol * an && rn <= fmax(tol, 1e-11)) ? 1 : 0;
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) w.lam[b * ld + i] = lam[i];
}

__global__ void ref_check_kernel(int nb, RefWork w, int k) {
  if (k > *w.rdone) return;
  int all = 1;
  for (int b = 0; b < nb; ++b) all &= w.conv[b];
  if (all) *w.rdone = k;
}

// Xf = the X after the last applied step (step g writes buffer (g + 1) % 2);
// no convergence within kRefMaxIt steps selects the Jacobi solver.
__global__ void ref_final_x_kernel(int ld, Pair2 nper, RefWork w) {
  const int b = blockIdx.y, n = nper.v[b];
  const int g = *w.rdone;
  const bool ok = g < kRefMaxIt;
  if (!ok && blockIdx.x == 0 && b == 0 && threadIdx.x == 0) *w.fallback = 1;
  const size_t sm = (size_t)ld * ld;
  const double2* X = (((ok ? g : kRefMaxIt - 1) + 1) % 2 == 0) ? w.X0 : w.X1;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n * n; e += gridDim.x * blockDim.x) {
    const int i = e / n, j = e % n;
    w.Xf[b * sm + (size_t)i * ld + j] = X[b * sm + (size_t)i * ld + j];
  }
}

// Clusters: the l_i of the last applied step sorted, consecutive values
// closer than its d grouped (so every pair that step left coupled lies in
// one cluster); each cluster's block of the final S = Xf^H A Xf is
// diagonalised by serial cyclic Jacobi (one thread per cluster).  Output per
// eigenpair P (sorted position of its cluster start s plus local index):
// ev[P] and cinfo[P] = (s, size, local, original index of sorted position P).
__global__ void ref_cluster_kernel(int ld, Pair2 nper, RefWork w) {
  __shared__ double dg[kRefMaxN];
  __shared__ int idx[kRefMaxN];
  __shared__ int cstart[kRefMaxN];
  const int b = blockIdx.x, n = nper.v[b];
  const size_t sm = (size_t)ld * ld;
  const double2* S = w.S + b * sm;
  if (*w.fallback) return;
  for (int i = threadIdx.x; i < n; i += blockDim.x) dg[i] = w.lam[(size_t)b * ld + i];
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    int r = 0;
    for (int j = 0; j < n; ++j) r += (dg[j] < dg[i]) || (dg[j] == dg[i] && j < i);
    idx[r] = i;
  }
  __syncthreads();
  const double tau = w.dlt[b];
  if (threadIdx.x == 0) {
    int s0 = 0;
    for (int p = 0; p < n; ++p) {
      if (p > 0 && dg[idx[p]] - dg[idx[p - 1]] > tau) s0 = p;
      cstart[p] = s0;
    }
  }
  __syncthreads();
  int* ci = w.cinfo + (size_t)b * ld * 4;
  double* ev = w.ev + (size_t)b * ld;
  double2* Qb = w.Q + (size_t)b * ld * kClusterMax;
  for (int p = threadIdx.x; p < n; p += blockDim.x) {
    if (cstart[p] != p) continue;            // one thread per cluster start
    int c = 1;
    while (p + c < n && cstart[p + c] == p) ++c;
    if (c > kClusterMax) {
      *w.fallback = 1;
      continue;
    }
    double2 a[kClusterMax][kClusterMax], q[kClusterMax][kClusterMax];
    for (int r = 0; r < c; ++r)
      for (int t = 0; t < c; ++t) {
        a[r][t] = S[(size_t)idx[p + r] * ld + idx[p + t]];
        q[r][t] = make_double2(r == t ? 1.0 : 0.0, 0.0);
      }
    double nrm = 0.0;
    for (int r = 0; r < c; ++r)
      for (int t = 0; t < c; ++t) nrm += a[r][t].x * a[r][t].x + a[r][t].y * a[r][t].y;
    nrm = sqrt(nrm);
    for (int sweep = 0; sweep < 40 && c > 1; ++sweep) {
      bool any = false;
      for (int r = 0; r < c; ++r)
        for (int t = r + 1; t < c; ++t) {
          const double2 apq = a[r][t];
          const double mag = hypot(apq.x, apq.y);
          if (mag <= 1e-300 || mag <= 2.220446049250313e-16 * 1e-2 * nrm) continue;
          any = true;
          const double app = a[r][r].x, aqq = a[t][t].x;
          const double theta = (aqq - app) / (2.0 * mag);
          double tt = 1.0 / (fabs(theta) + sqrt(theta * theta + 1.0));
          if (theta < 0.0) tt = -tt;
          const double cs = 1.0 / sqrt(tt * tt + 1.0), sn = tt * cs;
          // apq = mag e^{i phi}; G = [[cs, sn], [-sn e^{-i phi}, cs e^{-i phi}]] on (r, t)
          const double2 om = make_double2(apq.x / mag, -apq.y / mag);
          auto cm = [](double2 x, double2 y) { return make_double2(x.x * y.x - x.y * y.y, x.x * y.y + x.y * y.x); };
          for (int u = 0; u < c; ++u) {          // A <- A G, Q <- Q G (columns r, t)
            const double2 x0 = a[u][r], x1 = cm(a[u][t], om);
            a[u][r] = make_double2(cs * x0.x - sn * x1.x, cs * x0.y - sn * x1.y);
            a[u][t] = make_double2(sn * x0.x + cs * x1.x, sn * x0.y + cs * x1.y);
            const double2 y0 = q[u][r], y1 = cm(q[u][t], om);
            q[u][r] = make_double2(cs * y0.x - sn * y1.x, cs * y0.y - sn * y1.y);
            q[u][t] = make_double2(sn * y0.x + cs * y1.x, sn * y0.y + cs * y1.y);
          }
          const double2 oc = make_double2(om.x, -om.y);
          for (int u = 0; u < c; ++u) {          // A <- G^H A (rows r, t)
            const double2 x0 = a[r][u], x1 = cm(oc, a[t][u]);
            a[r][u] = make_double2(cs * x0.x - sn * x1.x, cs * x0.y - sn * x1.y);
            a[t][u] = make_double2(sn * x0.x + cs * x1.x, sn * x0.y + cs * x1.y);
          }
          a[r][t] = make_double2(0.0, 0.0);
          a[t][r] = make_double2(0.0, 0.0);
        }
      if (!any) break;
    }
    for (int l = 0; l < c; ++l) {
      ev[p + l] = a[l][l].x;
      int* cp = ci + (size_t)(p + l) * 4;
      cp[0] = p;
      cp[1] = c;
      cp[2] = l;
      for (int m = 0; m < c; ++m) Qb[(size_t)(p + m) * kClusterMax + l] = q[m][l];
    }
  }
  for (int pp = threadIdx.x; pp < n; pp += blockDim.x) ci[(size_t)pp * 4 + 3] = idx[pp];
}

// Acceptance test of the assembled pairs: with S = V^H A V and R = I - V^H V
// formed, any off-diagonal |S_ij| or diagonal |S_ii - w_i| above
// tol_s ||A||_F, or |R_ij| above tol_r, selects the Jacobi solver.
__global__ void ref_accept_kernel(int ld, Pair2 nper, RefWork w, const double* W, size_t sW, double tol_s,
                                  double tol_r) {
  __shared__ int bad;
  const int b = blockIdx.x, n = nper.v[b];
  if (*w.fallback) return;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  const size_t sm = (size_t)ld * ld;
  const double lim = tol_s * w.anorm[b];
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int i = e / n, j = e % n;
    double2 sv = w.S[b * sm + (size_t)i * ld + j];
    if (i == j) sv.x -= W[b * sW + i];
    const double2 rv = w.R[b * sm + (size_t)i * ld + j];
    if (!(hypot(sv.x, sv.y) <= lim) || !(hypot(rv.x, rv.y) <= tol_r)) bad = 1;
  }
  __syncthreads();
  if (threadIdx.x == 0 && bad) *w.fallback = 1;
}

// V[:, o(P)] = sum_m Xf[:, idx[s + m]] Q[s + m][l], w[o(P)] = ev[P], with o
// the ascending order of ev (ties by P).
__global__ void ref_assemble_kernel(int ld, Pair2 nper, RefWork w, double* W, size_t sW, double2* V, size_t sV) {
  __shared__ int opos[kRefMaxN];
  const int b = blockIdx.y, n = nper.v[b];
  if (*w.fallback) return;
  const size_t sm = (size_t)ld * ld;
  const double* ev = w.ev + (size_t)b * ld;
  const int* ci = w.cinfo + (size_t)b * ld * 4;
  for (int P = threadIdx.x; P < n; P += blockDim.x) {
    int r = 0;
    const double e = ev[P];
    for (int q = 0; q < n; ++q) r += (ev[q] < e) || (ev[q] == e && q < P);
    opos[P] = r;
    if (blockIdx.x == 0) W[b * sW + r] = e;
  }
  __syncthreads();
  const double2* X = w.Xf + b * sm;
  const double2* Qb = w.Q + (size_t)b * ld * kClusterMax;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n * n; e += gridDim.x * blockDim.x) {
    const int row = e / n, P = e % n;
    const int s0 = ci[(size_t)P * 4], c = ci[(size_t)P * 4 + 1], l = ci[(size_t)P * 4 + 2];
    double re = 0.0, im = 0.0;
    for (int m = 0; m < c; ++m) {
      const int col = ci[(size_t)(s0 + m) * 4 + 3];
      const double2 x = X[(size_t)row * ld + col], q = Qb[(size_t)(s0 + m) * kClusterMax + l];
      re += x.x * q.x - x.y * q.y;
      im += x.x * q.y + x.y * q.x;
    }
    V[b * sV + (size_t)row * ld + opos[P]] = make_double2(re, im);
  }
}

// ------------------------------------------------- Loewdin by Newton-Schulz --
// S^-1/2 from the coupled Newton-Schulz iteration on A = S / c, with c the
// largest absolute row sum (so the spectrum of A lies in (0, 1]):
//   T = (3 I - Z Y) / 2,  Y <- Y T,  Z <- T Z,   Y -> A^1/2, Z -> A^-1/2.
// This is the matrix the reference forms as V diag(w^-1/2) V^H
// (static.py:470-480) whenever no eigenvalue of S falls below its floor
// max(1e-12, eps max(w) n); S is then positive definite with condition far
// from that floor.  Steps after convergence are retired on the device.
constexpr int kNSMaxIt = 16;   // S is close to I after a gradient step: 4-6 steps in practice

// c_b and the start Y = S / c, Z = I; gate = large.
__global__ void ns_init_kernel(int ld, Pair2 nper, const double2* S, size_t sS, double2* Y, double2* Z, size_t sm,
                               double* cinv, int* gate) {
  const int b = blockIdx.x;
  const int n = nper.v[b];
  const double2* Sb = S + b * sS;
  __shared__ double red[32];
  double mx = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double rs = 0.0;
    for (int j = 0; j < n; ++j) {
      const double2 v = Sb[(size_t)i * ld + j];
      rs += hypot(v.x, v.y);
    }
    mx = fmax(mx, rs);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x / 32] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int w = 0; w < (int)(blockDim.x / 32); ++w) m = fmax(m, red[w]);
    red[0] = m;
    cinv[b] = 1.0 / m;
    if (b == 0) *gate = 1 << 30;
  }
  __syncthreads();
  const double ci = 1.0 / red[0];
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int i = e / n, j = e % n;
    const double2 v = Sb[(size_t)i * ld + j];
    Y[b * sm + (size_t)i * ld + j] = make_double2(v.x * ci, v.y * ci);
    Z[b * sm + (size_t)i * ld + j] = make_double2(i == j ? 1.0 : 0.0, 0.0);
  }
}

// After T of step k: if max|T - I| over both blocks is below 1e-9, step k
// is the last one applied (*gate = k); it squares that error to rounding.
__global__ void ns_check_kernel(int ld, Pair2 nper, const double2* T, size_t sm, int* gate, int k) {
  if (k > *gate) return;
  __shared__ double red[32];
  double mx = 0.0;
  for (int b = 0; b < 2; ++b) {
    const int n = nper.v[b];
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      const int i = e / n, j = e % n;
      const double2 v = T[b * sm + (size_t)i * ld + j];
      mx = fmax(mx, hypot(v.x - (i == j ? 1.0 : 0.0), v.y));
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x / 32] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int w = 0; w < (int)(blockDim.x / 32); ++w) m = fmax(m, red[w]);
    if (m < 1e-9) *gate = k;
  }
}

// U = Z_final / sqrt(c); the result of step k sits in buffer (k + 1) % 2.
__global__ void ns_final_kernel(int ld, Pair2 nper, const double2* Z0, const double2* Z1, size_t sm,
                                const double* cinv, const int* gate, double2* U, int* status) {
  const int b = blockIdx.y;
  const int n = nper.v[b];
  const int g = *gate;
  const bool ok = g < kNSMaxIt;
  const double2* Z = ((ok ? g : kNSMaxIt - 1) + 1) % 2 == 0 ? Z0 : Z1;
  const double sc = sqrt(cinv[b]);
  if (!ok && blockIdx.x == 0 && b == 0 && threadIdx.x == 0) latch_error(status, HFB_ERR_NO_CONVERGENCE);
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n * n; e += gridDim.x * blockDim.x) {
    const int i = e / n, j = e % n;
    const double2 v = Z[b * sm + (size_t)i * ld + j];
    U[b * sm + (size_t)i * ld + j] = make_double2(v.x * sc, v.y * sc);
  }
}

// Eigenpairs of up to two nearly diagonal Hermitian matrices (lower
// triangles at A + b sA, leading dimension ld): w ascending at W + b sW,
// eigenvectors in the columns of V + b sV; Jacobi when the refinement does
// not apply (see above).
static int eigh_refine(hfb_ctx_s* c, int nb, Pair2 nper, int ld, const double2* A, size_t sA, double* W, size_t sW,
                       double2* V, size_t sV, double tol_rel, cudaStream_t st) {
  if (ld > kRefMaxN) return HFB_ERR_UNSUPPORTED_GRID;
  const size_t sm = (size_t)ld * ld;
  const size_t bytes = sizeof(double2) * (8 * (size_t)nb * sm + (size_t)nb * ld * kClusterMax) +
                       sizeof(double) * (2 * (size_t)nb * ld + 2 * nb) + sizeof(int) * (nb + 2 + (size_t)nb * ld * 4) +
                       256;
  char* buf = (char*)scratch(c, hfb_ctx_s::S_EIG, bytes);
  if (!buf) return HFB_ERR_ALLOC;
  RefWork w;
  double2* mp = (double2*)buf;
  w.Ah = mp; w.X0 = mp + nb * sm; w.X1 = mp + 2 * nb * sm; w.AX = mp + 3 * nb * sm; w.S = mp + 4 * nb * sm;
  w.R = mp + 5 * nb * sm; w.E = mp + 6 * nb * sm; w.Xf = mp + 7 * nb * sm; w.Q = mp + 8 * nb * sm;
  double* dp = (double*)(w.Q + (size_t)nb * ld * kClusterMax);
  w.lam = dp; w.ev = dp + nb * ld; w.anorm = dp + 2 * nb * ld; w.dlt = w.anorm + nb;
  int* ip = (int*)(w.dlt + nb);
  w.conv = ip; w.rdone = ip + nb; w.fallback = ip + nb + 1; w.cinfo = ip + nb + 2;
  const double tol = tol_rel > 0.0 ? tol_rel : 1e-13;
  ref_init_kernel<<<nb, 1024, 0, st>>>(ld, nper, A, sA, w);
  HFB_CHECK_LAUNCH();
  int r;
  for (int k = 0; k < kRefMaxIt; ++k) {
    double2* Xc = (k % 2 == 0) ? w.X0 : w.X1;
    double2* Xn = (k % 2 == 0) ? w.X1 : w.X0;
    if ((r = zgemm_small(ld, ld, 0, 0, w.Ah, sm, Xc, sm, w.AX, sm, nper, nb, st, 1.0, 0.0, w.rdone, k))) return r;
    if ((r = zgemm_small(ld, ld, 1, 0, Xc, sm, w.AX, sm, w.S, sm, nper, nb, st, 1.0, 0.0, w.rdone, k))) return r;
    if ((r = zgemm_small(ld, ld, 1, 0, Xc, sm, Xc, sm, w.R, sm, nper, nb, st, -1.0, 1.0, w.rdone, k))) return r;
    ref_update_kernel<<<nb, 1024, 0, st>>>(ld, nper, w, k, tol);
    HFB_CHECK_LAUNCH();
    ref_check_kernel<<<1, 1, 0, st>>>(nb, w, k);
    HFB_CHECK_LAUNCH();
    if ((r = zgemm_small(ld, ld, 0, 0, Xc, sm, w.E, sm, Xn, sm, nper, nb, st, 1.0, 0.0, w.rdone, k))) return r;
  }
  ref_final_x_kernel<<<dim3(32, nb), 256, 0, st>>>(ld, nper, w);
  HFB_CHECK_LAUNCH();
  if ((r = zgemm_small(ld, ld, 0, 0, w.Ah, sm, w.Xf, sm, w.AX, sm, nper, nb, st))) return r;
  if ((r = zgemm_small(ld, ld, 1, 0, w.Xf, sm, w.AX, sm, w.S, sm, nper, nb, st))) return r;
  ref_cluster_kernel<<<nb, 256, 0, st>>>(ld, nper, w);
  HFB_CHECK_LAUNCH();
  ref_assemble_kernel<<<dim3(32, nb), 256, 0, st>>>(ld, nper, w, W, sW, V, sV);
  HFB_CHECK_LAUNCH();
  // accept only pairs that diagonalise A to the requested accuracy
  if ((r = zgemm_small(ld, ld, 0, 0, w.Ah, sm, V, sV, w.AX, sm, nper, nb, st))) return r;
  if ((r = zgemm_small(ld, ld, 1, 0, V, sV, w.AX, sm, w.S, sm, nper, nb, st))) return r;
  if ((r = zgemm_small(ld, ld, 1, 0, V, sV, V, sV, w.R, sm, nper, nb, st, -1.0, 1.0))) return r;
  ref_accept_kernel<<<nb, 1024, 0, st>>>(ld, nper, w, W, sW, fmax(1e3 * tol, 1e-11), fmax(1e3 * tol, 1e-11));
  HFB_CHECK_LAUNCH();
  // Jacobi for the cases the refinement leaves (runs only when *fallback)
  EighBatch eb{};
  eb.tol_rel = tol_rel;
  eb.gate = w.fallback;
  for (int b = 0; b < nb; ++b) {
    eb.n[eb.nb] = nper.v[b];
    eb.lda[eb.nb] = ld;
    eb.a[eb.nb] = A + b * sA;
    eb.w[eb.nb] = W + b * sW;
    eb.v[eb.nb] = V + b * sV;
    ++eb.nb;
  }
  return eigh_batch(c, eb, st);
}

// Y0, Z0, Y1, Z1, T: work matrices [2][ld][ld] each; S: [2] with stride sS.
static int loewdin_ns(hfb_ctx_s* c, int ld, Pair2 nper, const double2* S, size_t sS, double2* Y0, double2* Z0,
                      double2* Y1, double2* Z1, double2* T, double* cinv, int* gate, double2* U, cudaStream_t st) {
  const size_t sm = (size_t)ld * ld;
  ns_init_kernel<<<2, 256, 0, st>>>(ld, nper, S, sS, Y0, Z0, sm, cinv, gate);
  HFB_CHECK_LAUNCH();
  int r;
  for (int k = 0; k < kNSMaxIt; ++k) {
    double2* Yc = (k % 2 == 0) ? Y0 : Y1;
    double2* Zc = (k % 2 == 0) ? Z0 : Z1;
    double2* Yn = (k % 2 == 0) ? Y1 : Y0;
    double2* Zn = (k % 2 == 0) ? Z1 : Z0;
    if ((r = zgemm_small(ld, ld, 0, 0, Zc, sm, Yc, sm, T, sm, nper, 2, st, -0.5, 1.5, gate, k))) return r;
    ns_check_kernel<<<1, 1024, 0, st>>>(ld, nper, T, sm, gate, k);
    HFB_CHECK_LAUNCH();
    if ((r = zgemm_small(ld, ld, 0, 0, Yc, sm, T, sm, Yn, sm, nper, 2, st, 1.0, 0.0, gate, k))) return r;
    if ((r = zgemm_small(ld, ld, 0, 0, T, sm, Zc, sm, Zn, sm, nper, 2, st, 1.0, 0.0, gate, k))) return r;
  }
  ns_final_kernel<<<dim3(32, 2), 256, 0, st>>>(ld, nper, Z0, Z1, sm, cinv, gate, U, c->dev_status);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

// T = V diag(1/sqrt(max(w, thr))) with thr = max(1e-12, eps max(w) n) (static.py:473-479)
__global__ void loewdin_scale_kernel(int ld, Pair2 nper, const double* w, size_t sw, const double2* V,
                                     double2* T, size_t sm) {
  const int b = blockIdx.y;
  const int n = nper.v[b];
  const double* wb = w + b * sw;
  __shared__ double thr;
  if (threadIdx.x == 0) {
    double mx = wb[0];
    for (int k = 1; k < n; ++k) mx = fmax(mx, wb[k]);
    thr = fmax(1e-12, 2.220446049250313e-16 * mx * n);
  }
  __syncthreads();
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n * n; e += gridDim.x * blockDim.x) {
    const int i = e / n, j = e % n;
    const double s = 1.0 / sqrt(fmax(wb[j], thr));
    const double2 v = V[b * sm + (size_t)i * ld + j];
    T[b * sm + (size_t)i * ld + j] = make_double2(v.x * s, v.y * s);
  }
}

// Copy the diagonal's real part (sp_norm), and the lower-Hermitian lambda.
__global__ void diag_real_kernel(int ld, Pair2 nper, Pair2 off, const double2* S, size_t sm, double* out) {
  const int b = blockIdx.x;
  for (int k = threadIdx.x; k < nper.v[b]; k += blockDim.x) out[off.v[b] + k] = S[b * sm + (size_t)k * ld + k].x;
}

// construct_hfb_matrices after h, gap are in the new basis (static.py:511-575).
// One CTA per isospin.  H, G: [b][ld][ld]; writes hmatrix, gapmatrix,
// symcond, lambda_save [b][nmax][nmax], sp_energy, deltaf, efluct.
__global__ void __launch_bounds__(1024)
lambda_kernel(int ld, int nmax, Pair2 nper, Pair2 off, int ipair, int tbcs, const double2* H,
              const double2* G, size_t sm, const double* wocc, const double* wguv, const double* pairwg,
              const double* wstates, double2* hmat, double2* gmat, double2* symc, double2* lsave, double* sp_energy,
              double* deltaf, double* efluct) {
  const int b = blockIdx.x;
  const int n = nper.v[b], o = off.v[b];
  __shared__ double red_max[32], red_sum[32];
  const double2* Hb = H + b * sm;
  const double2* Gb = G + b * sm;
  double mx = 0.0, sm2 = 0.0;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int i = e / n, j = e % n;
    const double2 h = Hb[(size_t)i * ld + j];
    const double2 ht = Hb[(size_t)j * ld + i];
    double2 g = ipair ? Gb[(size_t)i * ld + j] : make_double2(0, 0);
    double2 gt = ipair ? Gb[(size_t)j * ld + i] : make_double2(0, 0);
    hmat[((size_t)b * nmax + i) * nmax + j] = h;
    if (tbcs && i != j) { g = make_double2(0, 0); }
    if (tbcs && i != j) { gt = make_double2(0, 0); }
    gmat[((size_t)b * nmax + i) * nmax + j] = g;
    // lambda_ij = w_j h_ij - wuv_j g_ij ; lambda^H_ij = conj(lambda_ji)
    const double wj = wocc[o + j] * wstates[o + j], wi = wocc[o + i] * wstates[o + i];
    const double uj = wguv[o + j] * pairwg[o + j] * wstates[o + j];
    const double ui = wguv[o + i] * pairwg[o + i] * wstates[o + i];
    const double2 l = make_double2(wj * h.x - uj * g.x, wj * h.y - uj * g.y);
    const double2 lt = make_double2(wi * ht.x - ui * gt.x, -(wi * ht.y - ui * gt.y));   // conj(lambda_ji)
    const double2 as = make_double2(0.5 * (l.x - lt.x), 0.5 * (l.y - lt.y));
    const double2 sy = make_double2(0.5 * (l.x + lt.x), 0.5 * (l.y + lt.y));
    symc[((size_t)b * nmax + i) * nmax + j] = as;
    lsave[((size_t)b * nmax + i) * nmax + j] = sy;
    const double ab = hypot(as.x, as.y);
    mx = fmax(mx, ab);
    sm2 += ab * ab;
  }
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    sp_energy[o + k] = Hb[(size_t)k * ld + k].x;
    if (ipair) deltaf[o + k] = Gb[(size_t)k * ld + k].x * pairwg[o + k];
  }
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, s));
    sm2 += __shfl_xor_sync(0xffffffffu, sm2, s);
  }
  if (threadIdx.x % 32 == 0) { red_max[threadIdx.x / 32] = mx; red_sum[threadIdx.x / 32] = sm2; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, s = 0;
    for (int k = 0; k < (int)(blockDim.x / 32); ++k) { a = fmax(a, red_max[k]); s += red_sum[k]; }
    efluct[b] = a;
    efluct[2 + b] = sqrt(s / ((double)n * n));
  }
}

// lsave [b][nmax][nmax] -> L [b][ld][ld] (lambda used for the Lagrange update)
__global__ void copy_lambda_kernel(int ld, int nmax, Pair2 nper, const double2* lsave, double2* L, size_t sm) {
  const int b = blockIdx.y;
  const int n = nper.v[b];
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n * n; e += gridDim.x * blockDim.x) {
    const int i = e / n, j = e % n;
    L[b * sm + (size_t)i * ld + j] = lsave[((size_t)b * nmax + i) * nmax + j];
  }
}

// ============================================================== rotate ====
// out1_j = sum_i psi_i U_ij, out2_j = sum_i psi_i L_ij for the states of one
// block: a (K x ns) by (ns x 2 ns) GEMM.  64 (k) x 64 (j) tile per CTA, 256
// threads with 4 x 4 outputs each, double-buffered 8-state stages.
template <class R>
__global__ void __launch_bounds__(256)
rotate_kernel(int ns, size_t K, const cplx<R>* __restrict__ psi, const double2* __restrict__ U,
              const double2* __restrict__ L, int ld, cplx<R>* out1, cplx<R>* out2) {
  using Z = cplx<R>;
  constexpr int KT = 64, JT = 64, IT = 8;
  __shared__ Z Ps[2][IT][KT + 1];
  __shared__ Z Ws[2][IT][JT + 1];
  const int njt = (2 * ns + JT - 1) / JT;
  const int jt = blockIdx.x % njt;
  const size_t k0 = (size_t)(blockIdx.x / njt) * KT;
  const int j0 = jt * JT;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;   // tx -> k (4), ty -> j (4)
  R acc[4][4][2];
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) acc[u][v][0] = acc[u][v][1] = R(0);
  auto load = [&](int buf, int i0) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int e = threadIdx.x + 256 * h;
      const int ii = e / KT, kk = e % KT;
      const size_t k = k0 + kk;
      Ps[buf][ii][kk] = (i0 + ii < ns && k < K) ? psi[(size_t)(i0 + ii) * K + k] : czero<Z>();
      const int ii2 = e / JT, jj = e % JT;
      const int j = j0 + jj;
      double2 w = make_double2(0, 0);
      if (i0 + ii2 < ns && j < 2 * ns)
        w = j < ns ? U[(size_t)(i0 + ii2) * ld + j] : L[(size_t)(i0 + ii2) * ld + (j - ns)];
      Ws[buf][ii2][jj] = mk<R>((R)w.x, (R)w.y);
    }
  };
  load(0, 0);
  __syncthreads();
  int buf = 0;
  for (int i0 = 0; i0 < ns; i0 += IT) {
    if (i0 + IT < ns) load(buf ^ 1, i0 + IT);
#pragma unroll
    for (int ii = 0; ii < IT; ++ii) {
      Z pv[4], wv[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) pv[u] = Ps[buf][ii][tx + 16 * u];
#pragma unroll
      for (int v = 0; v < 4; ++v) wv[v] = Ws[buf][ii][ty + 16 * v];
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          acc[u][v][0] += pv[u].x * wv[v].x - pv[u].y * wv[v].y;
          acc[u][v][1] += pv[u].x * wv[v].y + pv[u].y * wv[v].x;
        }
    }
    __syncthreads();
    buf ^= 1;
  }
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    const int j = j0 + ty + 16 * v;
    if (j >= 2 * ns) continue;
    Z* o = j < ns ? out1 + (size_t)j * K : out2 + (size_t)(j - ns) * K;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const size_t k = k0 + tx + 16 * u;
      if (k < K) o[k] = mk<R>(acc[u][v][0], acc[u][v][1]);
    }
  }
}

// FP64 states on the FP64 tensor cores (mma.sync m8n8k4 .f64): with the
// state index interleaved with (Re, Im), i' = 2 i + part,
//   A'[k][i'] = (Re, Im) psi_i(k),
//   Re out_j(k) = sum_i' A'[k][i'] Br[i'][j],  Br = (Re W_ij, -Im W_ij),
//   Im out_j(k) = sum_i' A'[k][i'] Bi[i'][j],  Bi = (Im W_ij,  Re W_ij),
// W = [U | L].  A CTA (8 warps, 4 along k x 2 along j, 32 x 32 outputs
// per warp, 4 x 4 MMA blocks) computes 128 grid points x 64 outputs,
// streaming the states in double-buffered stages of 4.
constexpr int RD_KT = 128, RD_JT = 64, RD_IT = 4;

__global__ void __launch_bounds__(256) rotate_dmma_kernel(int ns, size_t K, const double2* __restrict__ psi,
                                                          const double2* __restrict__ U,
                                                          const double2* __restrict__ L, int ld, double2* out1,
                                                          double2* out2) {
  __shared__ double2 Ps[2][RD_IT][RD_KT + 1];
  __shared__ double2 Ws[2][RD_IT][RD_JT + 1];
  const int njt = (2 * ns + RD_JT - 1) / RD_JT;
  const int jt = blockIdx.x % njt;
  const size_t k0 = (size_t)(blockIdx.x / njt) * RD_KT;
  const int j0 = jt * RD_JT;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wk = warp & 3, wj = warp >> 2;
  const int fr = lane >> 2, fk = lane & 3;
  double accR[4][4][2], accI[4][4][2];
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) accR[u][v][0] = accR[u][v][1] = accI[u][v][0] = accI[u][v][1] = 0.0;
  auto load = [&](int buf, int i0) {
    for (int e = threadIdx.x; e < RD_IT * RD_KT; e += 256) {
      const int ii = e / RD_KT, kk = e % RD_KT;
      const size_t k = k0 + kk;
      Ps[buf][ii][kk] = (i0 + ii < ns && k < K) ? psi[(size_t)(i0 + ii) * K + k] : make_double2(0.0, 0.0);
    }
    for (int e = threadIdx.x; e < RD_IT * RD_JT; e += 256) {
      const int ii = e / RD_JT, jj = e % RD_JT;
      const int j = j0 + jj;
      double2 w = make_double2(0.0, 0.0);
      if (i0 + ii < ns && j < 2 * ns)
        w = j < ns ? U[(size_t)(i0 + ii) * ld + j] : L[(size_t)(i0 + ii) * ld + (j - ns)];
      Ws[buf][ii][jj] = w;
    }
  };
  load(0, 0);
  __syncthreads();
  int buf = 0;
  for (int i0 = 0; i0 < ns; i0 += RD_IT) {
    if (i0 + RD_IT < ns) load(buf ^ 1, i0 + RD_IT);
#pragma unroll
    for (int kk = 0; kk < RD_IT / 2; ++kk) {
      const int ii = 2 * kk + (fk >> 1);     // state of this lane's k' within the step
      const bool im = fk & 1;
      double a[4], br[4], bi[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const double2 p = Ps[buf][ii][32 * wk + 8 * u + fr];
        a[u] = im ? p.y : p.x;
      }
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const double2 w = Ws[buf][ii][32 * wj + 8 * v + fr];
        br[v] = im ? -w.y : w.x;
        bi[v] = im ? w.x : w.y;
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          gd_mma(accR[u][v], a[u], br[v]);
          gd_mma(accI[u][v], a[u], bi[v]);
        }
    }
    __syncthreads();
    buf ^= 1;
  }
  // the thread holds rows k = 32 wk + 8 u + fr, columns j = 32 wj + 8 v + 2 fk + c
#pragma unroll
  for (int v = 0; v < 4; ++v)
#pragma unroll
    for (int c2 = 0; c2 < 2; ++c2) {
      const int j = j0 + 32 * wj + 8 * v + 2 * fk + c2;
      if (j >= 2 * ns) continue;
      double2* o = j < ns ? out1 + (size_t)j * K : out2 + (size_t)(j - ns) * K;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const size_t k = k0 + 32 * wk + 8 * u + fr;
        if (k < K) o[k] = make_double2(accR[u][v][c2], accI[u][v][c2]);
      }
    }
}

// Single-precision variant with a larger register tile: 128 (k) x 96 (j)
// per CTA, 256 threads holding 8 x 6 complex accumulators each (48
// independent chains), 8 states per double-buffered shared-memory stage.
// The 96-wide j tile keeps the padding of 2 ns columns small (280 -> 288,
// 192 -> 192).
constexpr int kRotKT = 128, kRotJT = 96, kRotIT = 8;

__global__ void __launch_bounds__(256, 1)
rotate_f32_kernel(int ns, size_t K, const float2* __restrict__ psi, const double2* __restrict__ U,
                  const double2* __restrict__ L, int ld, float2* out1, float2* out2) {
  __shared__ __align__(16) float2 Ps[2][kRotIT][kRotKT];
  __shared__ __align__(16) float2 Ws[2][kRotIT][kRotJT];
  const int njt = (2 * ns + kRotJT - 1) / kRotJT;
  const int jt = blockIdx.x % njt;
  const size_t k0 = (size_t)(blockIdx.x / njt) * kRotKT;
  const int j0 = jt * kRotJT;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;   // k = tx + 16 u (u < 8), j = ty + 16 v (v < 6)
  float acc[8][6][2];
#pragma unroll
  for (int u = 0; u < 8; ++u)
#pragma unroll
    for (int v = 0; v < 6; ++v) acc[u][v][0] = acc[u][v][1] = 0.f;
  // stage loads into registers first so the next stage's global reads
  // overlap this stage's arithmetic
  float4 pr[2];
  float2 wr[3];
  auto fetch = [&](int i0) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int e = threadIdx.x + 256 * h;          // 512 float4 = 8 states x 64 pairs
      const int ii = e / (kRotKT / 2), kk = 2 * (e % (kRotKT / 2));
      const size_t k = k0 + kk;
      pr[h] = make_float4(0.f, 0.f, 0.f, 0.f);
      if (i0 + ii < ns && k < K) {
        if (k + 2 <= K) pr[h] = *reinterpret_cast<const float4*>(psi + (size_t)(i0 + ii) * K + k);
        else { const float2 a = psi[(size_t)(i0 + ii) * K + k]; pr[h] = make_float4(a.x, a.y, 0.f, 0.f); }
      }
    }
#pragma unroll
    for (int h = 0; h < 3; ++h) {
      const int e = threadIdx.x + 256 * h;          // 768 = 8 states x 96 columns
      const int ii = e / kRotJT, jj = e % kRotJT;
      const int j = j0 + jj;
      double2 w = make_double2(0.0, 0.0);
      if (i0 + ii < ns && j < 2 * ns)
        w = j < ns ? U[(size_t)(i0 + ii) * ld + j] : L[(size_t)(i0 + ii) * ld + (j - ns)];
      wr[h] = make_float2((float)w.x, (float)w.y);
    }
  };
  auto stash = [&](int buf) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int e = threadIdx.x + 256 * h;
      const int ii = e / (kRotKT / 2), kk = 2 * (e % (kRotKT / 2));
      *reinterpret_cast<float4*>(&Ps[buf][ii][kk]) = pr[h];
    }
#pragma unroll
    for (int h = 0; h < 3; ++h) {
      const int e = threadIdx.x + 256 * h;
      Ws[buf][e / kRotJT][e % kRotJT] = wr[h];
    }
  };
  fetch(0);
  stash(0);
  __syncthreads();
  int buf = 0;
  for (int i0 = 0; i0 < ns; i0 += kRotIT) {
    const bool more = i0 + kRotIT < ns;
    if (more) fetch(i0 + kRotIT);
#pragma unroll
    for (int ii = 0; ii < kRotIT; ++ii) {
      float2 pv[8], wv[6];
#pragma unroll
      for (int u = 0; u < 8; ++u) pv[u] = Ps[buf][ii][tx + 16 * u];
#pragma unroll
      for (int v = 0; v < 6; ++v) wv[v] = Ws[buf][ii][ty + 16 * v];
#pragma unroll
      for (int u = 0; u < 8; ++u)
#pragma unroll
        for (int v = 0; v < 6; ++v) {
          acc[u][v][0] = fmaf(pv[u].x, wv[v].x, fmaf(-pv[u].y, wv[v].y, acc[u][v][0]));
          acc[u][v][1] = fmaf(pv[u].x, wv[v].y, fmaf(pv[u].y, wv[v].x, acc[u][v][1]));
        }
    }
    if (more) stash(buf ^ 1);
    __syncthreads();
    buf ^= 1;
  }
#pragma unroll
  for (int v = 0; v < 6; ++v) {
    const int j = j0 + ty + 16 * v;
    if (j >= 2 * ns) continue;
    float2* o = j < ns ? out1 + (size_t)j * K : out2 + (size_t)(j - ns) * K;
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const size_t k = k0 + tx + 16 * u;
      if (k < K) o[k] = make_float2(acc[u][v][0], acc[u][v][1]);
    }
  }
}

int rotate_tc_launch(hfb_ctx_s* c, int ns, const void* psi, const double2* U, const double2* L, int ld, void* out1,
                     void* out2, cudaStream_t st, int pre);   // rotate_tc.cu
int rotate_tc_transpose(hfb_ctx_s* c, int which, int ns, const void* psi, cudaStream_t st);

// ``pre`` (single precision on the tensor cores): 0 or 1 when the states were
// transposed already by rotate_tc_transpose into that rotation's buffer.
int rotate_launch(hfb_ctx_s* c, int prec, int s0, int ns, const void* psi, const double2* U, const double2* L, int ld,
                  void* out1, void* out2, cudaStream_t st, int pre) {
  if (ns <= 0) return HFB_OK;
  if (prec != HFB_F64 && c->use_tcgen05) {
    const size_t Kc = (size_t)2 * c->n * c->n * c->n, offc = (size_t)s0 * Kc;
    const int r = rotate_tc_launch(c, ns, (const float2*)psi + offc, U, L, ld, (float2*)out1 + offc,
                                   (float2*)out2 + offc, st, pre);
    if (r != HFB_ERR_UNSUPPORTED_GRID) return r;
  }
  const size_t K = (size_t)2 * c->n * c->n * c->n;
  const int njt = (2 * ns + 63) / 64;
  const size_t nkt = (K + 63) / 64;
  const size_t off = (size_t)s0 * K;
  if (prec == HFB_F64 && c->f64_mma) {
    const int njd = (2 * ns + RD_JT - 1) / RD_JT;
    const size_t nkd = (K + RD_KT - 1) / RD_KT;
    rotate_dmma_kernel<<<(unsigned)(nkd * njd), 256, 0, st>>>(ns, K, (const double2*)psi + off, U, L, ld,
                                                             (double2*)out1 + off, (double2*)out2 + off);
  } else if (prec == HFB_F64)
    rotate_kernel<double><<<(unsigned)(nkt * njt), 256, 0, st>>>(ns, K, (const double2*)psi + off, U, L, ld,
                                                                 (double2*)out1 + off, (double2*)out2 + off);
  else {
    const int njt2 = (2 * ns + kRotJT - 1) / kRotJT;
    const size_t nkt2 = (K + kRotKT - 1) / kRotKT;
    rotate_f32_kernel<<<(unsigned)(nkt2 * njt2), 256, 0, st>>>(ns, K, (const float2*)psi + off, U, L, ld,
                                                               (float2*)out1 + off, (float2*)out2 + off);
  }
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

}  // namespace hfb

using namespace hfb;

extern "C" int hfb_gram(hfb_ctx_t ctx, int prec, int s0, int ns, int mask, const void* psi, const void* hampsi,
                        const void* hmfpsi, const double* v_pair_iq, double wxyz, double* out, void* stream) {
  if (!ctx || !psi || !out || ns <= 0) return HFB_ERR_ARG;
  if (((mask & 2) && !hampsi) || ((mask & 4) && !hmfpsi) || ((mask & 8) && !v_pair_iq)) return HFB_ERR_ARG;
  if ((ns + GT - 1) / GT > 255) return HFB_ERR_ARG;
  double2* o = (double2*)out;
  double2* outs[8] = {o, o + (size_t)ns * ns, o + 2 * (size_t)ns * ns, o + 3 * (size_t)ns * ns,
                      nullptr, nullptr, nullptr, nullptr};
  const double* vp[2] = {v_pair_iq, nullptr};
  return gram_launch(ctx, prec, 1, &s0, &ns, &mask, psi, hampsi, hmfpsi, vp, wxyz, outs, ns, as_stream(stream));
}

extern "C" int hfb_eigh(hfb_ctx_t ctx, int nb, int n, int lda, const double* a, double* w, double* v, int* sweeps,
                        void* stream) {
  if (!ctx || !a || !w || !v || n <= 0 || lda < n) return HFB_ERR_ARG;
  return eigh_launch(ctx, nb, n, lda, (const double2*)a, w, (double2*)v, sweeps, as_stream(stream));
}

extern "C" int hfb_eigh_near_diagonal(hfb_ctx_t ctx, int nb, int n, int lda, const double* a, double* w,
                                      double* v, void* stream) {
  if (!ctx || !a || !w || !v || n <= 0 || lda < n || nb <= 0) return HFB_ERR_ARG;
  if (lda > kRefMaxN) return HFB_ERR_UNSUPPORTED_GRID;
  cudaStream_t st = as_stream(stream);
  const size_t mstride = (size_t)n * lda;
  for (int b0 = 0; b0 < nb; b0 += 2) {
    const int cnt = nb - b0 < 2 ? nb - b0 : 2;
    Pair2 nper;
    nper.v[0] = n;
    nper.v[1] = cnt > 1 ? n : 0;
    int r = eigh_refine(ctx, cnt, nper, lda, (const double2*)a + b0 * mstride, mstride, w + (size_t)b0 * n, n,
                        (double2*)v + b0 * mstride, mstride, 0.0, st);
    if (r) return r;
  }
  return HFB_OK;
}

extern "C" int hfb_diagstep(hfb_ctx_t ctx, int prec, const hfb_diag_args* a, void* stream) {
  if (!ctx || !a || !a->psi || !a->psi_out || a->psi_out == a->psi || !a->lagrange || !a->sp_norm || !a->lambda_save) return HFB_ERR_ARG;
  if (a->diagonalize && !a->hampsi) return HFB_ERR_ARG;
  if (a->construct && (!a->hmfpsi || !a->sp_energy || !a->hmatrix || !a->gapmatrix || !a->symcond || !a->efluct))
    return HFB_ERR_ARG;
  if (a->construct && a->ipair && (!a->v_pair || !a->deltaf)) return HFB_ERR_ARG;
  cudaStream_t st = as_stream(stream);
  const int n0 = a->npsi[0], n1 = a->npsi[1];
  const int ld = n0 > n1 ? n0 : n1;
  const size_t sm = (size_t)ld * ld;
  const size_t n3 = (size_t)ctx->n * ctx->n * ctx->n;
  // workspace: 4 Gram matrices + 10 work matrices per isospin, eigenvalues,
  // Newton-Schulz scalars
  const size_t nmat = 2 * (4 + 10);
  char* ws = (char*)scratch(ctx, hfb_ctx_s::S_SMALL,
                            sizeof(double2) * nmat * sm + sizeof(double) * 4 * ld + 8 * sizeof(double));
  if (!ws) return HFB_ERR_ALLOC;
  double2* gm = (double2*)ws;                 // [iq][4][ld][ld]: S, Lambda, H_old, G_old
  double2* Y0 = gm + 2 * 4 * sm;              // Newton-Schulz work
  double2* Z0 = Y0 + 2 * sm;
  double2* Y1 = Z0 + 2 * sm;
  double2* Z1 = Y1 + 2 * sm;
  double2* T = Z1 + 2 * sm;                   // scratch
  double2* Ur = T + 2 * sm;                   // S^-1/2
  double2* Vl = Ur + 2 * sm;                  // eigenvectors of lambda
  double2* U = Vl + 2 * sm;                   // total transform
  double2* Hn = U + 2 * sm;                   // U^H H U
  double2* Gn = Hn + 2 * sm;                  // U^H G U
  double2* Lw = Gn;                           // U lambda (Gn is dead by then)
  double* w = (double*)(Gn + 2 * sm);         // [iq][ld] (x2: unused, lambda)
  double* cinv = w + 4 * ld;
  int* gate = (int*)(cinv + 4);
  Pair2 nper, off;
  nper.v[0] = n0; nper.v[1] = n1;
  off.v[0] = 0; off.v[1] = n0;
  const int nq[2] = {n0, n1}, so[2] = {0, n0};
  int r;
  // The eigensolve of lambda runs on the side stream on a few SMs.  H and G
  // are needed only by the construct step after it, so when both are asked
  // for, the Gram launch computes S and lambda first and H, G follow on the
  // main stream while the eigensolve runs (HFB_GRAM_SPLIT=0: one launch).
  int mask = 1;
  if (a->diagonalize) mask |= 2;
  if (a->construct) mask |= 4;
  if (a->construct && a->ipair) mask |= 8;
  const bool split = a->diagonalize && a->construct && ctx->side && ctx->gram_split;
  const double* vp[2] = {a->v_pair, a->v_pair ? a->v_pair + n3 : nullptr};
  double2* outs[8];
  for (int iq = 0; iq < 2; ++iq)
    for (int m = 0; m < 4; ++m) outs[iq * 4 + m] = gm + ((size_t)iq * 4 + m) * sm;
  {
    const int m1 = split ? (mask & 3) : mask;
    const int masks[2] = {m1, m1};
    r = gram_launch(ctx, prec, 2, so, nq, masks, a->psi, a->hampsi, a->hmfpsi, vp, a->wxyz, outs, ld, st);
    if (r) return r;
  }
  diag_real_kernel<<<2, 256, 0, st>>>(ld, nper, off, gm, 4 * sm, a->sp_norm);
  HFB_CHECK_LAUNCH();
  // Newton-Schulz needs S only: with the split Gram it runs on a second side
  // stream, beside the H, G launch and the eigensolve, on the SMs they leave
  const bool ns_side = split && ctx->side2;
  cudaStream_t nst = st;
  if (ns_side) {
    cudaEventRecord(ctx->ev_fork2, st);
    cudaStreamWaitEvent(ctx->side2, ctx->ev_fork2, 0);
    nst = ctx->side2;
  }
  // eigh of lambda (Jacobi, one CTA per isospin, or the refinement) on the
  // side stream while the main stream runs the H, G Gram launch (or, without
  // the split, the Newton-Schulz GEMMs for S^-1/2)
  const bool fork = a->diagonalize && ctx->side;
  if (a->diagonalize) {
    cudaStream_t es = st;
    if (fork) {
      cudaEventRecord(ctx->ev_fork, st);
      cudaStreamWaitEvent(ctx->side, ctx->ev_fork, 0);
      es = ctx->side;
    }
    // single-precision states carry rounding noise of 2^-24 relative in
    // lambda; converging below that level refines nothing
    const double tol_rel = prec != HFB_F64 ? 5.9604644775390625e-08 : 0.0;
    // FP64: refinement (measured 1 ms per Pb208 iteration faster than the
    // Jacobi sweeps near convergence); FP32: the looser Jacobi threshold
    // converges in a few sweeps and measured faster (11.4 ms against 12.0
    // ms per Pb208 iteration: in the bulk the refinement's acceptance test
    // fails and the Jacobi runs after it)
    if (ctx->lambda_refine && prec == HFB_F64) {
      r = eigh_refine(ctx, 2, nper, ld, gm + sm, 4 * sm, w + 2 * ld, ld, Vl, sm, tol_rel, es);
    } else {
      EighBatch eb{};
      eb.tol_rel = tol_rel;
      for (int iq = 0; iq < 2; ++iq) {
        eb.n[eb.nb] = nq[iq];
        eb.lda[eb.nb] = ld;
        eb.a[eb.nb] = gm + (size_t)iq * 4 * sm + sm;
        eb.w[eb.nb] = w + 2 * ld + (size_t)iq * ld;
        eb.v[eb.nb] = Vl + (size_t)iq * sm;
        ++eb.nb;
      }
      r = eigh_batch(ctx, eb, es);
    }
    if (r) return r;
    if (fork) cudaEventRecord(ctx->ev_join, ctx->side);
  }
  if (split) {
    const int m2 = mask & 12;
    const int masks[2] = {m2, m2};
    r = gram_launch(ctx, prec, 2, so, nq, masks, a->psi, a->hampsi, a->hmfpsi, vp, a->wxyz, outs, ld, st);
    if (r) return r;
  }
  r = loewdin_ns(ctx, ld, nper, gm, 4 * sm, Y0, Z0, Y1, Z1, T, cinv, gate, Ur, nst);
  if (r) return r;
  // the rotation's transposes of the states depend on psi only: they follow
  // Newton-Schulz on the second side stream
  int pre[2] = {-1, -1};
  if (ns_side && prec != HFB_F64 && ctx->use_tcgen05) {
    const size_t Kc = (size_t)2 * n3;
    for (int iq = 0; iq < 2; ++iq) {
      r = rotate_tc_transpose(ctx, iq, nq[iq], (const float2*)a->psi + (size_t)so[iq] * Kc, nst);
      if (r == HFB_OK) pre[iq] = iq;
      else if (r != HFB_ERR_UNSUPPORTED_GRID) return r;
    }
  }
  if (ns_side) {
    cudaEventRecord(ctx->ev_join2, ctx->side2);
    cudaStreamWaitEvent(st, ctx->ev_join2, 0);
  }
  double2* Uuse = Ur;
  if (a->diagonalize) {
    if (fork) cudaStreamWaitEvent(st, ctx->ev_join, 0);
    r = zgemm_small(ld, ld, 0, 0, Ur, sm, Vl, sm, U, sm, nper, 2, st);
    if (r) return r;
    Uuse = U;
  }
  const int nmax = a->nmax;
  if (a->construct) {
    // H = U^H (H_old U), G likewise
    r = zgemm_small(ld, ld, 0, 0, gm + 2 * sm, 4 * sm, Uuse, sm, T, sm, nper, 2, st);
    if (r) return r;
    r = zgemm_small(ld, ld, 1, 0, Uuse, sm, T, sm, Hn, sm, nper, 2, st);
    if (r) return r;
    if (a->ipair) {
      r = zgemm_small(ld, ld, 0, 0, gm + 3 * sm, 4 * sm, Uuse, sm, T, sm, nper, 2, st);
      if (r) return r;
      r = zgemm_small(ld, ld, 1, 0, Uuse, sm, T, sm, Gn, sm, nper, 2, st);
      if (r) return r;
    }
    lambda_kernel<<<2, 1024, 0, st>>>(ld, nmax, nper, off, a->ipair, a->tbcs, Hn, Gn, sm, a->wocc, a->wguv, a->pairwg,
                                      a->wstates, (double2*)a->hmatrix, (double2*)a->gapmatrix, (double2*)a->symcond,
                                      (double2*)a->lambda_save, a->sp_energy, a->deltaf, a->efluct);
    HFB_CHECK_LAUNCH();
  }
  // L = U lambda_save (lambda_save just written when construct)
  copy_lambda_kernel<<<dim3(64, 2), 256, 0, st>>>(ld, nmax, nper, (const double2*)a->lambda_save, T, sm);
  HFB_CHECK_LAUNCH();
  r = zgemm_small(ld, ld, 0, 0, Uuse, sm, T, sm, Lw, sm, nper, 2, st);
  if (r) return r;
  for (int iq = 0; iq < 2; ++iq) {
    r = rotate_launch(ctx, prec, so[iq], nq[iq], a->psi, Uuse + (size_t)iq * sm, Lw + (size_t)iq * sm, ld, a->psi_out,
                      a->lagrange, st, pre[iq]);
    if (r) return r;
  }
  return HFB_OK;
}
