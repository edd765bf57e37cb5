"""Restart files (hfb.restart): the format round trip on host tensors, the
checks on mismatched states, and (GPU) a run continued from a file."""
import os
import types

import numpy as np
import pytest
import torch


def _fake_state(n=8, npsi=(3, 2), dtype=torch.complex128, seed=0, iteration=17):
    g = torch.Generator().manual_seed(seed)
    ns = npsi[0] + npsi[1]
    r = lambda *s: torch.randn(*s, generator=g, dtype=torch.float64)
    lv = types.SimpleNamespace(nneut=4, nprot=2, npsi=npsi, psi=torch.complex(r(ns, 2, n, n, n), r(ns, 2, n, n, n)).to(dtype))
    for k in ("sp_energy", "sp_norm", "wocc", "wguv", "pairwg", "wstates", "deltaf"):
        setattr(lv, k, r(ns))
    dens = types.SimpleNamespace(rho=r(2, n, n, n), tau=r(2, n, n, n), chi=r(2, n, n, n), current=r(2, 3, n, n, n),
                                 sdens=r(2, 3, n, n, n), sodens=r(2, 3, n, n, n))
    grids = types.SimpleNamespace(nx=n, ny=n, nz=n, dx=0.8, dy=0.8, dz=0.8)
    params = types.SimpleNamespace(iteration=iteration, trestart=False)
    return dict(levels=lv, densities=dens, grids=grids, params=params)


def _zeroed(st):
    z = _fake_state(seed=1, iteration=0)
    for k in ("psi", "sp_energy", "sp_norm", "wocc", "wguv", "pairwg", "wstates", "deltaf"):
        getattr(z["levels"], k).zero_()
    for k in ("rho", "tau", "chi", "current", "sdens", "sodens"):
        getattr(z["densities"], k).zero_()
    return z


def test_restart_round_trip(tmp_path):
    from hfb import restart
    st = _fake_state()
    p = os.path.join(tmp_path, "s.hfbr")
    restart.save_state(p, st)
    hdr = restart.read_header(p)
    assert hdr["iteration"] == 17 and hdr["npsi"] == [3, 2]
    assert all(m["offset"] % 64 == 0 for m in hdr["arrays"].values())
    z = _zeroed(st)
    restart.load_state(p, z)
    assert z["params"].iteration == 17 and z["params"].trestart
    for k in ("psi", "sp_energy", "wocc", "deltaf"):
        assert torch.equal(getattr(z["levels"], k), getattr(st["levels"], k)), k
    for k in ("rho", "current", "sodens"):
        assert torch.equal(getattr(z["densities"], k), getattr(st["densities"], k)), k


def test_restart_precision_change_and_mismatch(tmp_path):
    from hfb import restart
    st = _fake_state(dtype=torch.complex64)
    p = os.path.join(tmp_path, "s.hfbr")
    restart.save_state(p, st)
    assert restart.read_header(p)["arrays"]["psi"]["dtype"] == "complex64"
    z = _zeroed(st)                                     # complex128 target
    restart.load_state(p, z)
    assert torch.equal(z["levels"].psi, st["levels"].psi.to(torch.complex128))
    bad = _zeroed(st)
    bad["grids"].dx = 0.9
    with pytest.raises(ValueError, match="grid"):
        restart.load_state(p, bad)
    bad = _zeroed(st)
    bad["levels"].nneut = 6
    with pytest.raises(ValueError, match="nucleus"):
        restart.load_state(p, bad)
    with open(p, "r+b") as f:
        f.write(b"NOTHFBRS")
    with pytest.raises(ValueError, match="not an hfb restart"):
        restart.read_header(p)


@pytest.mark.gpu
def test_run_continued_from_restart_file(tmp_path):
    """O16 on 16^3 (the golden run case): 20 iterations, save, load into a
    fresh state, continue with the reference's restart semantics; the
    continued run converges to the energy of an uninterrupted run."""
    import copy
    from hfb import config, static, restart
    from cases import RUN_CASES

    def setup():
        return config.setup(copy.deepcopy(RUN_CASES["o16_n16"]))

    st = setup()
    static.statichf(**st, maxiter=20)
    p = os.path.join(tmp_path, "o16.hfbr")
    restart.save_state(p, st)
    e20 = st["energies"].ehf
    st2 = setup()
    restart.load_state(p, st2)
    assert st2["params"].iteration == 20
    _, res = static.statichf(**st2, maxiter=400, de_tol=1e-10)
    assert res.history[0]["iteration"] == 20 and res.history[1]["iteration"] == 21
    assert abs(res.history[0]["ehf"] - e20) < 0.5       # starts where the first run stopped
    _, res3 = static.statichf(**setup(), maxiter=400, de_tol=1e-10)
    assert abs(res.history[-1]["ehf"] - res3.history[-1]["ehf"]) < 1e-6
