"""The oracle's vector-Jacobian products of hpsi and of the densities
(oracle/vjp.py) against central differences of the oracle's own hpsi01 and
density terms, on the CPU.  hpsi is linear in psi and in each field and the
densities are quadratic in psi, so central differences are exact up to
rounding and the bar is 1e-9 relative.  Anisotropic spacings, per-state
weights and both pairing terms are on."""
import copy

import numpy as np
import pytest

from oracle import model, meanfield as omf, densities as od, vjp

N, D = 8, (0.9, 1.0, 1.1)
NAMES = ("rho", "chi", "tau", "current", "sdens", "sodens")


def _rc(rng, *s):
    return rng.standard_normal(s) + 1j * rng.standard_normal(s)


@pytest.fixture(scope="module")
def setup():
    rng = np.random.default_rng(7)
    g = model.init_grids(N, N, N, *D)
    ns = 4
    mf = omf.init_meanfield(g)
    for k in ("upot", "bmass", "v_pair"):
        getattr(mf, k)[:] = rng.standard_normal((2, N, N, N))
    for k in ("aq", "spot", "wlspot"):
        getattr(mf, k)[:] = rng.standard_normal((2, 3, N, N, N))
    return dict(rng=rng, g=g, mf=mf, psi=_rc(rng, ns, 2, N, N, N), yb=_rc(rng, ns, 2, N, N, N),
                v=_rc(rng, ns, 2, N, N, N), w=rng.uniform(0.2, 1.0, ns), wu=rng.uniform(0.0, 0.5, ns))


def _close(a, b):
    assert abs(a - b) <= 1e-9 * max(abs(a), abs(b), 1.0), (a, b)


@pytest.mark.parametrize("iq", [0, 1])
def test_hpsi_vjp_matches_central_differences(setup, iq):
    s = setup
    g, mf, psi, yb, v, w, wu = (s[k] for k in ("g", "mf", "psi", "yb", "v", "w", "wu"))

    def L(m, x):
        return np.sum((np.conj(yb) * omf.hpsi01(g, m, iq, w, wu, x)[0]).real)

    pb, bars = vjp.hpsi_vjp(g, mf, iq, w, wu, psi, yb)
    e = 1e-3
    _close(np.sum((np.conj(pb) * v).real), (L(mf, psi + e * v) - L(mf, psi - e * v)) / (2 * e))
    for k, b in bars.items():
        Q = s["rng"].standard_normal(b.shape)
        mp, mm = copy.deepcopy(mf), copy.deepcopy(mf)
        getattr(mp, k)[iq] += e * Q
        getattr(mm, k)[iq] -= e * Q
        _close(np.sum(b * Q), (L(mp, psi) - L(mm, psi)) / (2 * e))


@pytest.mark.parametrize("iq", [0, 1])
def test_densities_vjp_matches_central_differences(setup, iq):
    s = setup
    g, psi, v, w, wu = (s[k] for k in ("g", "psi", "v", "w", "wu"))
    F = [x.sum(axis=0) for x in od.state_contributions(w, wu, psi, g.d)]
    fb = {nm: s["rng"].standard_normal(x.shape) for nm, x in zip(NAMES, F)}

    def L(x):
        return sum(np.sum(fb[nm] * y.sum(axis=0)) for nm, y in zip(NAMES, od.state_contributions(w, wu, x, g.d)))

    pb = vjp.densities_vjp(g, w, wu, psi, iq, fb)
    e = 1e-3
    _close(np.sum((np.conj(pb) * v).real), (L(psi + e * v) - L(psi - e * v)) / (2 * e))
