// Step-size control and energy history on the device, so that a run of
// self-consistent iterations can be replayed (a CUDA graph) without the host
// reading anything in between.  One thread, after the energies of an
// iteration:
//   hist[count] = E_bind, count += 1 (while count < max)
//   and, with the adaptation on, the rule of static.py:1864-1878:
//     x0 *= 1.005 if (E < E_prev and efluct1 < efluct1_prev (1 - 1e-5))
//                  or efluct2 < efluct2_prev (1 - 1e-5), else x0 *= 0.8;
//     x0 = min(max(x0, x0_min), 5 x0_min); the previous values updated,
// with efluct1 = max over the isospins, efluct2 their mean
// (static.py:574-575), from the diagonalisation step's fluctuations.
#include "hfb_ctx.cuh"

namespace hfb {
namespace {

__global__ void step_control_kernel(const double* __restrict__ ehf, const double* __restrict__ efluct, double* ctl,
                                    double* hist, int* count, int max_hist) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double e = *ehf;
  const int k = *count;
  if (k < max_hist) {
    hist[k] = e;
    *count = k + 1;
  }
  if (ctl[5] != 0.0) {
    const double ef1 = fmax(efluct[0], efluct[1]);
    const double ef2 = 0.5 * (efluct[2] + efluct[3]);
    double x0 = ctl[0];
    if ((e < ctl[1] && ef1 < ctl[2] * (1.0 - 1.0e-5)) || ef2 < ctl[3] * (1.0 - 1.0e-5))
      x0 *= 1.005;
    else
      x0 *= 0.8;
    x0 = fmin(fmax(x0, ctl[4]), 5.0 * ctl[4]);
    ctl[0] = x0;
    ctl[1] = e;
    ctl[2] = ef1;
    ctl[3] = ef2;
  }
}

}  // namespace
}  // namespace hfb

using namespace hfb;

extern "C" int hfb_step_control(hfb_ctx_t ctx, const double* ehf, const double* efluct, double* ctl, double* hist,
                                int* count, int max_hist, void* stream) {
  if (!ctx || !ehf || !efluct || !ctl || !hist || !count || max_hist < 0) return HFB_ERR_ARG;
  step_control_kernel<<<1, 32, 0, as_stream(stream)>>>(ehf, efluct, ctl, hist, count, max_hist);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}
