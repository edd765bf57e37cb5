"""Reverse-mode derivatives of hpsi and of the densities, as
torch.autograd.Functions over the library's kernels.

The reference gets these from JAX's reverse mode through hpsi01
(meanfield.py:41-159) and the density terms (densities.py:237-330).  Here
they follow from two exact properties of those discretisations:

* h is Hermitian, and the bilinear form <a|h[P]|b> is the integral of each
  potential field times the matching pair density of (a, b) -- upot: rho,
  bmass: tau, v_pair: 2 chi, aq: current, spot: sdens, wlspot: sodens --
  plus, for bmass, the Nyquist term of cderv02 (levels.py:314-330).  The
  pair densities come from the density kernel by polarisation,
  F(a, b) = (F(a + b) - F(a - b)) / 4, each pair first balanced in norm.
* The densities are quadratic forms in psi, so their VJP is 2 w h[F_bar] psi
  (+ wu chi_bar psi) with the Nyquist term of the tau cotangent removed.

VJP of y = w h psi - wu v_pair psi:
    psi_bar = w h ybar - wu v_pair ybar,
    P_bar   = sum_s w_s F_s(ybar_s, psi_s) for each field (v_pair: -2 wu chi),
    bmass_bar additionally the Nyquist pair term (hfb_nyquist_pair).
VJP of the densities:
    psi_bar = hpsi with fields (rho_bar, tau_bar, chi_bar, current_bar,
              sdens_bar, sodens_bar), weights (2 w, -wu), minus the Nyquist
              term of tau_bar (hfb_nyquist_apply).

Complex gradients follow torch's convention, dL = Re sum conj(x.grad) dx.
States are [nst][2][nx][ny][nz], neutrons first (``nneut`` of them); fields
are per isospin, [2][...].
"""
import torch

from ._lib import call, ptr, stream_ptr, prec_of
from .densities import init_densities
from .meanfield import init_meanfield

_FIELDS = ("upot", "bmass", "v_pair", "aq", "spot", "wlspot")
_DENS = ("rho", "chi", "tau", "current", "sdens", "sodens")


def _vec(x, nst, dev):
    return torch.as_tensor(x, dtype=torch.float64, device=dev).reshape(-1).expand(nst).contiguous()


def _densities(grids, psi, nneut, w, wu):
    """Densities of ``psi`` with occupation weights w and pairing weights wu."""
    nst = psi.shape[0]
    d = init_densities(grids)
    one = torch.ones(nst, dtype=torch.float64, device=psi.device)
    call("hfb_add_density", grids.ctx.handle, prec_of(psi), nst, nneut, ptr(psi), ptr(w), ptr(wu), ptr(one), ptr(one),
         1.0, ptr(d.rho), ptr(d.chi), ptr(d.tau), ptr(d.current), ptr(d.sdens), ptr(d.sodens), None, None,
         stream_ptr())
    return d


def _axpby_diag(grids, a, x, b, y):
    call("hfb_state_axpby_diag", grids.ctx.handle, prec_of(x), x.shape[0], ptr(a), ptr(x), float(b), ptr(y),
         stream_ptr())


def pair_densities(grids, a, b, nneut, w, wu):
    """sum_s w_s F(a_s, b_s) for rho, tau, current, sdens, sodens and
    sum_s wu_s chi(a_s, b_s), the pair densities Re(a^dagger O_F b), by
    polarisation of the density kernel (each pair balanced in norm)."""
    nst = a.shape[0]
    na = torch.linalg.vector_norm(a.reshape(nst, -1), dim=1).double()
    nb = torch.linalg.vector_norm(b.reshape(nst, -1), dim=1).double()
    ok = (na > 0) & (nb > 0)
    s = torch.where(ok, torch.sqrt(nb / torch.where(ok, na, torch.ones_like(na))), torch.ones_like(na)).contiguous()
    inv = (1.0 / s).contiguous()
    p = torch.zeros_like(a)
    m = torch.zeros_like(a)
    _axpby_diag(grids, s, a, 0.0, p)       # p = s a
    _axpby_diag(grids, s, a, 0.0, m)
    _axpby_diag(grids, inv, b, 1.0, p)     # p = s a + b / s
    _axpby_diag(grids, -inv, b, 1.0, m)    # m = s a - b / s
    dp = _densities(grids, p, nneut, w, wu)
    dm = _densities(grids, m, nneut, w, wu)
    return {k: (getattr(dp, k) - getattr(dm, k)) * 0.25 for k in _DENS}


def _pack(grids, fields, dtype):
    """A Meanfield whose fields are ``fields`` (missing ones zero), packed."""
    mf = init_meanfield(grids, dtype)
    for k, v in fields.items():
        getattr(mf, k).copy_(v)
    return mf.pack(dtype)


def _hpsi(grids, pot, x, nneut, w, wu):
    out = torch.empty_like(x)
    call("hfb_hpsi", grids.ctx.handle, prec_of(x), ptr(pot), x.shape[0], nneut, ptr(x), ptr(w), ptr(wu), ptr(out),
         None, None, stream_ptr())
    return out


def hpsi_vjp(grids, pot, psi, nneut, w, wu, ybar):
    """(psi_bar, {field: cotangent}) for y = w h psi - wu v_pair psi."""
    nst = psi.shape[0]
    psi_bar = _hpsi(grids, pot, ybar.contiguous(), nneut, w, wu)
    pd = pair_densities(grids, ybar.contiguous(), psi, nneut, w, wu)
    bmass = pd["tau"].clone()
    call("hfb_nyquist_pair", grids.ctx.handle, prec_of(psi), nst, nneut, ptr(ybar.contiguous()), ptr(psi), ptr(w),
         ptr(bmass), stream_ptr())
    bars = dict(upot=pd["rho"], bmass=bmass, v_pair=-2.0 * pd["chi"], aq=pd["current"], spot=pd["sdens"],
                wlspot=pd["sodens"])
    return psi_bar, bars


def densities_vjp(grids, psi, nneut, w, wu, bars):
    """psi_bar for cotangents ``bars`` (dict over rho, chi, tau, current,
    sdens, sodens; missing ones zero) of the densities of psi."""
    f = dict(upot=bars.get("rho"), bmass=bars.get("tau"), v_pair=bars.get("chi"), aq=bars.get("current"),
             spot=bars.get("sdens"), wlspot=bars.get("sodens"))
    mf = _pack(grids, {k: v for k, v in f.items() if v is not None}, psi.dtype)
    w2 = (2.0 * w).contiguous()
    out = _hpsi(grids, mf.pot, psi, nneut, w2, (-wu).contiguous())
    tau = bars.get("tau")
    if tau is not None:
        tmp = out.clone()
        call("hfb_nyquist_apply", grids.ctx.handle, prec_of(psi), psi.shape[0], nneut, ptr(tau.contiguous()), ptr(w2),
             ptr(psi), ptr(tmp), stream_ptr())
        out = tmp
    return out


class HPsi(torch.autograd.Function):
    """y = w h[fields] psi - wu v_pair psi (meanfield.py:41-159, both
    isospins: states below ``nneut`` use the neutron fields), differentiable
    in psi and in the six potential fields (each [2][...], float64)."""

    @staticmethod
    def forward(ctx, psi, upot, bmass, v_pair, aq, spot, wlspot, grids, nneut, weight=1.0, weightuv=0.0):
        psi = psi.contiguous()
        nst = psi.shape[0]
        w, wu = _vec(weight, nst, psi.device), _vec(weightuv, nst, psi.device)
        fields = dict(upot=upot, bmass=bmass, v_pair=v_pair, aq=aq, spot=spot, wlspot=wlspot)
        mf = _pack(grids, fields, psi.dtype)
        ctx.save_for_backward(psi, mf.pot, w, wu)
        ctx.grids, ctx.nneut = grids, nneut
        return _hpsi(grids, mf.pot, psi, nneut, w, wu)

    @staticmethod
    def backward(ctx, ybar):
        psi, pot, w, wu = ctx.saved_tensors
        psi_bar, bars = hpsi_vjp(ctx.grids, pot, psi, ctx.nneut, w, wu, ybar.contiguous())
        return (psi_bar,) + tuple(bars[k] for k in _FIELDS) + (None, None, None, None)


class Densities(torch.autograd.Function):
    """(rho, chi, tau, current, sdens, sodens) of psi (densities.py:177-330)
    with per-state weights w = wocc * wstates and wu = wguv * pairwg *
    wstates, differentiable in psi."""

    @staticmethod
    def forward(ctx, psi, grids, nneut, weight=1.0, weightuv=0.0):
        psi = psi.contiguous()
        nst = psi.shape[0]
        w, wu = _vec(weight, nst, psi.device), _vec(weightuv, nst, psi.device)
        d = _densities(grids, psi, nneut, w, wu)
        ctx.save_for_backward(psi, w, wu)
        ctx.grids, ctx.nneut = grids, nneut
        return tuple(getattr(d, k) for k in _DENS)

    @staticmethod
    def backward(ctx, *grads):
        psi, w, wu = ctx.saved_tensors
        bars = {k: g.contiguous() for k, g in zip(_DENS, grads) if g is not None}
        return densities_vjp(ctx.grids, psi, ctx.nneut, w, wu, bars), None, None, None, None


def hpsi(psi, fields, grids, nneut, weight=1.0, weightuv=0.0):
    """Differentiable hpsi; ``fields`` a dict over upot, bmass, v_pair, aq,
    spot, wlspot (float64 tensors [2][...] / [2][3][...])."""
    return HPsi.apply(psi, *(fields[k] for k in _FIELDS), grids, nneut, weight, weightuv)


def densities(psi, grids, nneut, weight=1.0, weightuv=0.0):
    """Differentiable densities: dict over rho, chi, tau, current, sdens, sodens."""
    return dict(zip(_DENS, Densities.apply(psi, grids, nneut, weight, weightuv)))
