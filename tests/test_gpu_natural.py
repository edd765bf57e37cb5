"""Device hfb_natural (configuration-space sub-iterations) against the
reference's own function (golden vectors, its index ranges, pairing off) and
against the oracle's restatement on the isospins' whole blocks.  FP64 states
and matrices: 1e-11 relative (max |diff| / max |ref|)."""
import os
import types

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from conftest import GOLDEN  # noqa: E402

TOL = 1e-11


def rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _device_state(d, tag):
    import hfb
    g = hfb.grids.init_grids(hfb.params.init_params(), nx=8, ny=8, nz=8, dx=0.9, dy=0.9, dz=0.9)
    T = lambda k: torch.from_numpy(np.ascontiguousarray(d[f"{tag}_in_{k}"])).cuda()   # noqa: E731
    lv = types.SimpleNamespace(nneut=3, nprot=2, npsi=[4, 3], nstmax=7)
    for k in ("psi", "lagrange", "sp_energy", "wocc", "wguv", "pairwg", "wstates", "deltaf"):
        setattr(lv, k, T(k))
    lv.psi_spare = torch.zeros_like(lv.psi)
    st = types.SimpleNamespace(e0bas=10.0 if tag == "e0" else 0.0, delstepbas=2.0)
    for k in ("hmatrix", "gapmatrix", "symcond", "lambda_save"):
        setattr(st, k, T(k))
    forces = types.SimpleNamespace(ipair=0)
    return g, lv, st, forces


@pytest.mark.parametrize("tag", ["e0", "glob"])
def test_natural_matches_reference(tag):
    import hfb
    d = dict(np.load(os.path.join(GOLDEN, "natural_n8.npz")))
    g, lv, st, forces = _device_state(d, tag)
    for iq in range(2):
        hfb.static.hfb_natural(forces, g, lv, None, None, st, iq, 3, reference_indexing=True)
    for k in ("psi", "lagrange", "sp_energy"):
        assert rel(getattr(lv, k), d[f"{tag}_out_{k}"]) < TOL, k
    for k in ("hmatrix", "gapmatrix", "symcond", "lambda_save"):
        assert rel(getattr(st, k), d[f"{tag}_out_{k}"]) < TOL, k


@pytest.mark.parametrize("tag", ["e0", "glob"])
def test_natural_whole_blocks_match_oracle(tag):
    import hfb
    from oracle import static as ost
    d = dict(np.load(os.path.join(GOLDEN, "natural_n8.npz")))
    g, lv, st, forces = _device_state(d, tag)
    lvo = types.SimpleNamespace(nneut=3, nprot=2, npsi=[4, 3], nstmax=7)
    for k in ("psi", "lagrange", "sp_energy", "wocc", "wguv", "pairwg", "wstates", "deltaf"):
        setattr(lvo, k, d[f"{tag}_in_{k}"].copy())
    sto = types.SimpleNamespace(e0bas=st.e0bas, delstepbas=2.0)
    for k in ("hmatrix", "gapmatrix", "symcond", "lambda_save"):
        setattr(sto, k, d[f"{tag}_in_{k}"].copy())
    for iq in range(2):
        hfb.static.hfb_natural(forces, g, lv, None, None, st, iq, 4)
        ost.hfb_natural(lvo, sto, iq, 4)
    for k in ("psi", "lagrange", "sp_energy"):
        assert rel(getattr(lv, k), getattr(lvo, k)) < TOL, k
    for k in ("hmatrix", "gapmatrix", "symcond", "lambda_save"):
        assert rel(getattr(st, k), getattr(sto, k)) < TOL, k


def test_driver_with_sub_iterations_matches_oracle():
    """The loop with configuration-space sub-iterations and pairing between
    them (VDI pairing, HFB weights after iteration 4, three sub-iterations
    per isospin from iteration 7) follows the oracle's loop, which calls its
    restated hfb_natural at the same place (static.py:1796-1798), on the
    oracle's own step-size schedule: E_bind per iteration to 1e-7 MeV."""
    import copy
    import hfb
    from cases import RUN_CASES
    from oracle import static as ost
    case = copy.deepcopy(RUN_CASES["ne20_vdi_n16"])
    case["force"]["tbcs"] = False
    case["static"].update(maxiter=12, inibcs=4, inidiag=4, iternat=3, iternat_start=6)
    rs = ost.build(copy.deepcopy(case))
    ost.prepare(rs)
    for i in range(1, 13):
        ost.iterate(rs, i)
    sched = [0.0] + [h["x0dmp"] for h in rs.history]
    st = hfb.config.setup(case)
    _, res = hfb.static.statichf(**st, maxiter=12, x0_schedule=sched)
    e_gpu = np.array([h["ehf"] for h in res.history[1:]])
    e_ora = np.array([h["ehf"] for h in rs.history])
    assert np.max(np.abs(e_gpu - e_ora)) < 1e-7
