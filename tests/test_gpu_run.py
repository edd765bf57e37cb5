"""End-to-end parity of the CUDA iteration with the reference driver.

The three golden runs were produced by the reference's own
statichf_with_benchmark (tests/golden/make_golden.py); the CUDA path replays
the recorded step-size schedule (see hfb.static.iterate) and must match the
per-iteration E_bind to 1e-7 MeV in FP64, and the final densities, levels,
Fermi energies and radii.  The FP32 path with an FP64 refinement tail must
land within 1 keV of the reference's E_bind.
"""
import copy
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from conftest import GOLDEN  # noqa: E402
from cases import RUN_CASES  # noqa: E402


def rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _sorted(v, npsi):
    v = v.detach().cpu().numpy() if isinstance(v, torch.Tensor) else np.asarray(v)
    return np.concatenate([np.sort(v[:npsi[0]]), np.sort(v[npsi[0]:])])


def _setup(name, dtype=torch.complex128):
    import hfb
    case = copy.deepcopy(RUN_CASES[name])
    return hfb.config.setup(case, dtype=dtype)


@pytest.mark.parametrize("name", sorted(RUN_CASES))
def test_fp64_run_matches_reference(name):
    import hfb
    ref = dict(np.load(os.path.join(GOLDEN, f"run_{name}.npz")))
    st = _setup(name)
    assert rel(st["levels"].psi, ref["psi0"]) < 1e-13
    out, res = hfb.static.statichf(**st, x0_schedule=ref["hist_x0dmp"])
    h = res.history
    assert abs(h[0]["ehf"] - ref["hist_ehf"][0]) < 1e-8
    ehf = np.array([r["ehf"] for r in h[1:]])
    ehfint = np.array([r["ehfint"] for r in h[1:]])
    ef2 = np.array([r["efluct2"] for r in h[1:]])
    np.testing.assert_allclose(ehf, ref["hist_ehf"][1:], rtol=0, atol=1e-7)
    np.testing.assert_allclose(ehfint, ref["hist_ehfint"][1:], rtol=0, atol=1e-7)
    np.testing.assert_allclose(ef2, ref["hist_efluct2"][1:], rtol=1e-5, atol=1e-11)
    dens, lv, pairs = st["densities"], st["levels"], st["pairs"]
    assert rel(dens.rho, ref["rho"]) < 1e-8
    assert rel(dens.tau, ref["tau"]) < 1e-8
    assert rel(_sorted(lv.sp_energy, lv.npsi), _sorted(ref["sp_energy"], lv.npsi)) < 1e-8
    if RUN_CASES[name]["force"]["ipair"] != 0:
        assert rel(dens.chi, ref["chi"]) < 1e-7
        assert rel(pairs.eferm, ref["eferm"]) < 1e-8
        assert rel(_sorted(lv.wocc, lv.npsi), _sorted(ref["wocc"], lv.npsi)) < 1e-7
    pnr, rms, rmstot = hfb.output.rms_radii(dens, st["grids"])
    assert np.max(np.abs(np.array(rms) - ref["rms"])) < 1e-9
    assert abs(st["energies"].ehf - float(ref["ehf"])) < 1e-7
    # deformation of the final state against the reference's observables
    obs = dict(np.load(os.path.join(GOLDEN, "observables_n16.npz")))
    o = hfb.output.calculate_complete_observables(dens, lv, st["grids"])
    assert abs(o.rmstot - float(obs[f"{name}_rmstot"])) < 1e-9
    assert np.max(np.abs(o.q20 - obs[f"{name}_q20"])) < 1e-6
    assert abs(o.beta - float(obs[f"{name}_beta"])) < 1e-8


@pytest.mark.parametrize("name", ["o16_n16", "ne20_vdi_n16"])
def test_fp32_with_fp64_tail_within_1kev(name):
    """Bulk iterations in FP32 (complex64 states) then an FP64 tail: E_bind
    within 1 keV of the reference's FP64 run on the same schedule."""
    import hfb
    ref = dict(np.load(os.path.join(GOLDEN, f"run_{name}.npz")))
    st = _setup(name, dtype=torch.complex64)
    n = RUN_CASES[name]["static"]["maxiter"]
    tail = 6
    (_, _, en, *_), res = hfb.static.statichf(**st, maxiter=n - tail, x0_schedule=ref["hist_x0dmp"])
    hfb.static.to_precision(st, torch.complex128)
    for i in range(n - tail + 1, n + 1):
        hfb.static.iterate(i, **{k: st[k] for k in ("coulomb", "densities", "energies", "forces", "grids",
                                                   "levels", "meanfield", "params", "static", "pairs")},
                           x0_schedule=ref["hist_x0dmp"])
    assert abs(st["energies"].ehf - float(ref["ehf"])) < 1e-3
