// Internal launch helpers shared between translation units.
#pragma once
#include "hfb_ctx.cuh"

namespace hfb {

// hpsi on states [s0, s0+ns): ``acc`` receives / accumulates h psi and may
// alias pout_mf or pout.  ``ovl`` (optional) receives per-state partial sums
// [ns][hpsi_ovl_parts][2] of Re<psi|h psi> and Re<psi|pout> (without wxyz).
int hpsi_launch(hfb_ctx_s* c, int prec, const void* pot, int s0, int ns, int nneut, const void* psi,
                const double* weight, const double* weightuv, void* acc, void* pout, void* pout_mf, void* pout_del,
                double* ovl, cudaStream_t st);

// Single-precision hpsi on the tensor cores (hpsi_tc.cu): derivative
// matrices built at context creation, availability, the launch (same
// contract as hpsi_launch) and its number of overlap partials per state.
int hpsi_tc_prepare(hfb_ctx_s* c);
bool hpsi_tc_available(hfb_ctx_s* c, int prec);
int hpsi_tc_parts(hfb_ctx_s* c);
int hpsi_tc_launch(hfb_ctx_s* c, const void* pot, int s0, int ns, int nneut, const void* psi, const double* weight,
                   const double* weightuv, void* acc, void* pout, void* pout_mf, void* pout_del, double* ovl,
                   cudaStream_t st);

// The same on the bf16 three-term kernel (hpsi_bf3.cu), two CTAs per SM.
int hpsi_bf3_prepare(hfb_ctx_s* c);
bool hpsi_bf3_available(hfb_ctx_s* c, int prec);
int hpsi_bf3_parts(hfb_ctx_s* c);
int hpsi_bf3_launch(hfb_ctx_s* c, const void* pot, int s0, int ns, int nneut, const void* psi, const double* weight,
                    const double* weightuv, void* acc, void* pout, void* pout_mf, void* pout_del, double* ovl,
                    cudaStream_t st);

// Double-precision hpsi on the FP64 tensor cores (hpsi_dmma.cu): the
// derivative matrices in double, built at context creation; same contract
// and overlap partials (one per y-plane) as the FFT kernels.
int hpsi_dmma_prepare(hfb_ctx_s* c);
bool hpsi_dmma_available(hfb_ctx_s* c, int prec);
int hpsi_dmma_launch(hfb_ctx_s* c, const void* pot, int s0, int ns, int nneut, const void* psi, const double* weight,
                     const double* weightuv, void* acc, void* pout, void* pout_mf, void* pout_del, double* ovl,
                     cudaStream_t st);

// Partial sums per state that hpsi_launch writes into ``ovl``.
int hpsi_ovl_parts(hfb_ctx_s* c, int prec);

// (E0+T)^-1 preconditioner (levels.py:398-437) on states [0, ns):
//  v = src - (use_lag ? lag : coef[s] * psi)     (plain src if psi == NULL)
//  out = F^-1[ F[v] / (denom(k) * Ntot) ]       (unnormalised transforms)
//  mode 0: dst = out;  mode 1: dst -= x0 * out   (dst = psi in the gradient step)
// ``tmp`` holds the intermediate spectrum (may alias src or dst).  ``x0_dev``
// (optional) is a device double read in place of x0.
// ``fluct`` (optional) receives per-(state, x-plane) partial sums [ns][n][2]
// of |v|^2 and |lag - coef psi|^2.  ``wg``, ``wu`` are per-state weights
// before the max(., 0.1) floor; the pairing shift uses vmax_dev[iq] when
// given, else vmax_host.
int precond_launch(hfb_ctx_s* c, int prec, int ns, int nneut, const void* src, const void* lag, int use_lag,
                   const void* psi, const double* coef, const double* wg, const double* wu, const double* vmax_dev,
                   double vmax_host, double e0, double h2ma, int mode, double x0, void* tmp, void* dst,
                   double* fluct, cudaStream_t st, const double* x0_dev = nullptr);

}  // namespace hfb
