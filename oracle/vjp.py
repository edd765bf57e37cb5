"""Vector-Jacobian products of hpsi and of the densities (oracle; test
infrastructure).

The reference differentiates these maps with JAX's reverse mode through
meanfield.py:41-159 (hpsi01) and densities.py:237-330 (the per-state
density terms).  Restated here from two exact identities of those
discretisations:

* h is Hermitian, and for every potential field P_F of hpsi01 the bilinear
  form <a|h[P]|b> is the integral of P_F times the matching density of the
  pair (a, b): upot <-> rho, aq <-> current, spot <-> sdens, wlspot <->
  sodens, v_pair <-> 2 chi (chi carries a factor 1/2), and bmass <-> tau
  plus the Nyquist term of cderv02 (levels.py:314-330): per line along
  each axis, -c mean(B) Re(conj(a_N) b_N) with a_N = sum_j (-1)^j a_j and
  c = -(pi/d)^2 / n.
* The pair density is the polarisation of the quadratic one,
  F(a, b) = (F(a + b) - F(a - b)) / 4.

So the VJP of y = w h psi - wu v_pair psi is psi_bar = w h ybar - wu
v_pair ybar, with field cotangents the pair densities of (ybar, psi); and
the VJP of the densities is psi_bar = 2 w h[F_bar] psi + wu chi_bar psi
with the Nyquist term of tau removed (the density tau has none).
Convention: dL = Re sum conj(x_bar) dx, the one torch uses for complex
tensors.
"""
import numpy as np

from . import densities as od
from . import meanfield as omf


def _pair_densities(psi, ybar, w, wu, d):
    """Sum over states of w_s (resp. wu_s for chi) times the pair densities
    of (ybar_s, psi_s), by polarisation; each pair is balanced in norm first."""
    na = np.sqrt(np.sum(np.abs(psi) ** 2, axis=(1, 2, 3, 4)))
    nb = np.sqrt(np.sum(np.abs(ybar) ** 2, axis=(1, 2, 3, 4)))
    a = np.sqrt(np.where(na > 0, nb / np.where(na > 0, na, 1.0), 1.0))
    a = np.where(a > 0, a, 1.0)[:, None, None, None, None]
    p, q = psi * a, ybar / a
    fp = od.state_contributions(w, wu, p + q, d)
    fm = od.state_contributions(w, wu, p - q, d)
    return [((x - y) / 4.0).sum(axis=0) for x, y in zip(fp, fm)]


def nyquist_pair(grids, a, b, w):
    """Field sum_axes (pi/d)^2 / n^2 sum_s w_s Re(conj(a_N) b_N) (per line,
    the same value at every point of the line): the cotangent of bmass from
    the Nyquist term of cderv02."""
    n = grids.nx
    out = np.zeros((n, n, n))
    e = (-1.0) ** np.arange(n)
    for ax in range(3):
        sh = [1] * 5
        sh[2 + ax] = n
        aN = np.sum(a * e.reshape(sh), axis=2 + ax)
        bN = np.sum(b * e.reshape(sh), axis=2 + ax)
        m = np.einsum("s,s...->...", w, (np.conj(aN) * bN).real.sum(axis=1))
        out = out + (np.pi / grids.d[ax]) ** 2 / n ** 2 * np.expand_dims(m, ax)
    return out


def nyquist_apply(grids, field, scale, x):
    """sum_axes c mean_line(field) (-1)^j x_N on every state (c = -(pi/d)^2/n),
    scaled per state: the Nyquist term of cderv02 with B = field."""
    n = grids.nx
    out = np.zeros_like(x)
    e = (-1.0) ** np.arange(n)
    for ax in range(3):
        sh = [1] * 5
        sh[2 + ax] = n
        xN = np.sum(x * e.reshape(sh), axis=2 + ax, keepdims=True)
        fm = np.mean(field, axis=ax, keepdims=True)[None, None]
        c = -(np.pi / grids.d[ax]) ** 2 / n
        out = out + c * fm * xN * e.reshape(sh)
    return out * np.asarray(scale)[:, None, None, None, None]


def hpsi_vjp(grids, mf, iq, weight, weightuv, psi, ybar):
    """VJP of y = hpsi01(grids, mf, iq, weight, weightuv, psi)[0] (states of
    one isospin).  Returns (psi_bar, dict of field cotangents for isospin iq:
    upot, bmass, v_pair, aq, spot, wlspot)."""
    ns = psi.shape[0]
    w = np.broadcast_to(np.asarray(weight, dtype=np.float64), (ns,))
    wu = np.broadcast_to(np.asarray(weightuv, dtype=np.float64), (ns,))
    psi_bar = omf.hpsi01(grids, mf, iq, w, wu, ybar)[0]
    rho, chi, tau, cur, sd, so = _pair_densities(psi, ybar, w, wu, grids.d)
    bars = dict(upot=rho, bmass=tau + nyquist_pair(grids, ybar, psi, w), v_pair=-2.0 * chi, aq=cur, spot=sd,
                wlspot=so)
    return psi_bar, bars


def densities_vjp(grids, weight, weightuv, psi, iq, bars):
    """VJP of the per-isospin sums of state_contributions (states of one
    isospin) for the cotangents ``bars`` (rho, chi, tau, current, sdens,
    sodens of that isospin).  Returns psi_bar."""
    ns = psi.shape[0]
    w = np.broadcast_to(np.asarray(weight, dtype=np.float64), (ns,))
    wu = np.broadcast_to(np.asarray(weightuv, dtype=np.float64), (ns,))
    mf = omf.init_meanfield(grids)
    mf.upot[iq] = bars["rho"]
    mf.bmass[iq] = bars["tau"]
    mf.v_pair[iq] = bars["chi"]
    mf.aq[iq] = bars["current"]
    mf.spot[iq] = bars["sdens"]
    mf.wlspot[iq] = bars["sodens"]
    out = omf.hpsi01(grids, mf, iq, 2.0 * w, -wu, psi)[0]
    return out + nyquist_apply(grids, bars["tau"], 2.0 * w, psi)
