"""Accuracy of the mixed-precision driver against the plain FP64 run on the
Cr48 workload (32^3, dx 0.8 fm, 32 + 32 states, volume delta pairing,
deformed oscillator start): single-precision bulk on the tensor cores, FP64
refinement tail.  Targets: |dE_bind| <= 1 keV, |d r_rms(p)| <= 1e-4 fm,
max |d e_i| <= 1e-3 MeV over the single-particle energies."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _spe(st):
    lv = st["levels"]
    e = lv.sp_energy.detach().cpu().numpy()
    n0 = lv.npsi[0]
    return np.concatenate([np.sort(e[:n0]), np.sort(e[n0:])])


def test_mixed_matches_fp64_on_cr48():
    from hfb import config, static
    from hfb.output import rms_radii
    case = config.case_dict("Cr48")
    st64 = config.setup(case, dtype=torch.complex128)
    S = {k: st64[k] for k in static._STATE_KEYS}
    static.prepare(**S)
    E = []
    for i in range(1, 3001):
        static.iterate(i, **S)
        E.append(st64["energies"].ehf)
        rem = static.remaining_change(E)
        if i > 60 and rem is not None and abs(rem) < 5e-6:
            break
    st32 = config.setup(case, dtype=torch.complex64)
    hist, sw = static.statichf_mixed(st32, maxiter=3000, stop_mev=5e-6)
    assert sw is not None and hist[-1][2] == "f64"
    assert abs(hist[-1][1] - E[-1]) <= 1e-3
    _, r32, _ = rms_radii(st32["densities"], st32["grids"])
    _, r64, _ = rms_radii(st64["densities"], st64["grids"])
    assert abs(r32[1] - r64[1]) <= 1e-4
    assert np.max(np.abs(_spe(st32) - _spe(st64))) <= 1e-3
