// Post-convergence quasiparticle spectrum: lastdiag (static.py:1072-1168).
//
// In the basis of the converged states of one isospin block the HFB matrix
// is assembled from the h and gap matrices left by the last diagonalisation
// step and the BCS occupations w_i (static.py:1093-1124):
//     H_ij = (h_ij - eferm delta_ij) xi_ij + gap_ij eta_ij,
//     xi_ij  = -sqrt(w_i w_j) + sqrt((1 - w_i)(1 - w_j)),
//     eta_ij =  sqrt(w_i (1 - w_j)) + sqrt(w_j (1 - w_i)),
// a Hermitian matrix (h, gap Hermitian; xi, eta symmetric).  Its eigenvalues
// (ascending) are the quasiparticle energies; the lower-component norm of
// eigenvector j is || C V[:, j] || with the sparse coefficient matrix of
// static.py:1129-1139, which couples each state to its time-reversal
// partner by the parity of its index within the whole state array:
//     C[i][i-1] = -sqrt(w_i)   (global index of i even),
//     C[i][i+1] =  sqrt(w_i)   (global index of i odd),
// entries whose partner falls outside the block omitted.
// The eigenvectors come from the library's FP64 cyclic Jacobi solver.
#include <math.h>
#include "hfb_ctx.cuh"

namespace hfb {

int eigh_launch(hfb_ctx_s* c, int nb, int n, int lda, const double2* a, double* w, double2* v, int* sweeps,
                cudaStream_t st);   // diag.cu

namespace {

__global__ void lastdiag_assemble_kernel(int nst, int ldh, const double2* __restrict__ h,
                                         const double2* __restrict__ gap, const double* __restrict__ w,
                                         const double* __restrict__ eferm, double2* __restrict__ m) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nst * nst) return;
  const int i = e / nst, j = e % nst;
  const double wi = w[i], wj = w[j];
  const double xi = -sqrt(wi * wj) + sqrt((1.0 - wi) * (1.0 - wj));
  const double eta = sqrt(wi * (1.0 - wj)) + sqrt(wj * (1.0 - wi));
  double2 hv = h[(size_t)i * ldh + j];
  if (i == j) hv.x -= *eferm;
  const double2 g = gap[(size_t)i * ldh + j];
  m[e] = make_double2(hv.x * xi + g.x * eta, hv.y * xi + g.y * eta);
}

// One thread per eigenvector j: sum over components i of |(C V)[i][j]|^2
// in increasing i (the order of static.py:1144-1148).
__global__ void lastdiag_norm_kernel(int nst, int first, const double* __restrict__ w, const double2* __restrict__ v,
                                     double* __restrict__ qpn) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nst) return;
  double s = 0.0;
  for (int i = 0; i < nst; ++i) {
    const int gi = first + i;
    double2 l = make_double2(0.0, 0.0);
    if ((gi & 1) == 0 && i >= 1) {
      const double cf = -sqrt(w[i]);
      const double2 x = v[(size_t)(i - 1) * nst + j];
      l = make_double2(cf * x.x, cf * x.y);
    } else if ((gi & 1) == 1 && i + 1 < nst) {
      const double cf = sqrt(w[i]);
      const double2 x = v[(size_t)(i + 1) * nst + j];
      l = make_double2(cf * x.x, cf * x.y);
    }
    s += l.x * l.x + l.y * l.y;
  }
  qpn[j] = sqrt(s);
}

}  // namespace
}  // namespace hfb

extern "C" int hfb_lastdiag(hfb_ctx_t ctx, int nst, int ldh, const double* hmatrix, const double* gapmatrix,
                            const double* wocc, const double* eferm, int first, double* qp_energy, double* qp_norm,
                            void* stream) {
  using namespace hfb;
  if (!ctx || !hmatrix || !gapmatrix || !wocc || !eferm || !qp_energy || !qp_norm) return HFB_ERR_ARG;
  if (nst <= 0 || ldh < nst || first < 0) return HFB_ERR_ARG;
  cudaStream_t st = as_stream(stream);
  const size_t mm = (size_t)nst * nst;
  double2* m = (double2*)scratch(ctx, hfb_ctx_s::S_LAST, 2 * mm * sizeof(double2));
  if (!m) return HFB_ERR_ALLOC;
  double2* v = m + mm;
  lastdiag_assemble_kernel<<<(unsigned)((mm + 255) / 256), 256, 0, st>>>(
      nst, ldh, (const double2*)hmatrix, (const double2*)gapmatrix, wocc, eferm, m);
  HFB_CHECK_LAUNCH();
  int r = eigh_launch(ctx, 1, nst, nst, m, qp_energy, v, nullptr, st);
  if (r) return r;
  lastdiag_norm_kernel<<<(unsigned)((nst + 127) / 128), 128, 0, st>>>(nst, first, wocc, v, qp_norm);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}
