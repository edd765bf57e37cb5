"""Sensitivities of the self-consistent binding energy to the Skyrme
couplings and the pairing strengths.

At a converged HF-BCS solution E_bind is stationary with respect to the
single-particle states (under orthonormality) and the BCS occupations (at
fixed particle number), so the adjoint variable of the fixed-point map
vanishes for the energy and its total derivative is the explicit one:

    dE/dtheta = sum_b  dE/db (fixed densities) * db/dtheta
                + dE/dpower + dE/dv0_q,

with dE/db the integrals that multiply each coefficient in the integrated
functional (energies.py:117-258; computed on the device by
``hfb_energy_grad``), db/dtheta from forces.py:95-107, and, for the
volume / density-dependent delta pairing (meanfield.py:368-382), a pairing
energy linear in v0_q: dE/dv0_q = -epair_q / v0_q (pairs.py:116-126, the
pairing energy enters E_bind with a minus sign, energies.py:313-315).

Parameters (``PARAMS``): the eleven Skyrme couplings of the force table
(forces.py:60-107) t0-t3, x0-x3, t4 (the spin-orbit strength W0 as it
enters b4 = t4/2), b4p (the isovector spin-orbit coefficient, independent
of t4 in the table) and power (alpha), then v0neut, v0prot.  ``W0`` is also
accepted: the direction that moves t4 and b4p in proportion (SLy4's b4 =
b4p = W0/2 together), the coupling the parameter sweep perturbs.

``coupling_gradient(state)`` evaluates the gradient on a converged state;
``converge`` runs a state to a tight energy tolerance; ``fd_gradient`` is the
central finite-difference check; ``BindingEnergy`` puts the pair behind a
torch.autograd.Function (forward = self-consistent solve at theta, backward
= the explicit gradient above).
"""
import copy
import ctypes as C
import math

import numpy as np
import torch

from . import config, static
from ._lib import call, ptr, stream_ptr, HFB_F64

SKYRME = ("t0", "t1", "t2", "t3", "x0", "x1", "x2", "x3", "t4", "b4p", "power")
PARAMS = SKYRME + ("v0neut", "v0prot")
_B = ("b0", "b0p", "b1", "b1p", "b2", "b2p", "b3", "b3p", "b4", "b4p")


def b_gradient(state):
    """dE/db (b0 .. b4p) and dE/dpower at fixed densities, as a dict."""
    d, g, f = state["densities"], state["grids"], state["forces"]
    out = torch.zeros(11, dtype=torch.float64, device="cuda")
    call("hfb_energy_grad", g.ctx.handle, f.c_struct(), ptr(d.rho), ptr(d.tau), ptr(d.current), ptr(d.sdens),
         ptr(d.sodens), ptr(out), stream_ptr())
    v = out.cpu().numpy()
    res = dict(zip(_B, v[:10]))
    res["power"] = float(v[10])
    return res


def _db_dtheta(f):
    """Partial derivatives of the b coefficients (forces.py:95-107) with
    respect to each coupling, as {theta: {b: value}}."""
    t0, t1, t2, t3, t4 = f.t0, f.t1, f.t2, f.t3, f.t4
    x0, x1, x2, x3 = f.x0, f.x1, f.x2, f.x3
    return {
        "t0": {"b0": 1.0 + 0.5 * x0, "b0p": 0.5 + x0},
        "x0": {"b0": 0.5 * t0, "b0p": t0},
        "t1": {"b1": (1.0 + 0.5 * x1) / 4.0, "b1p": (0.5 + x1) / 4.0,
               "b2": 3.0 * (1.0 + 0.5 * x1) / 8.0, "b2p": 3.0 * (0.5 + x1) / 8.0},
        "x1": {"b1": t1 / 8.0, "b1p": t1 / 4.0, "b2": 3.0 * t1 / 16.0, "b2p": 3.0 * t1 / 8.0},
        "t2": {"b1": (1.0 + 0.5 * x2) / 4.0, "b1p": -(0.5 + x2) / 4.0,
               "b2": -(1.0 + 0.5 * x2) / 8.0, "b2p": (0.5 + x2) / 8.0},
        "x2": {"b1": t2 / 8.0, "b1p": -t2 / 4.0, "b2": -t2 / 16.0, "b2p": t2 / 8.0},
        "t3": {"b3": (1.0 + 0.5 * x3) / 4.0, "b3p": (0.5 + x3) / 4.0},
        "x3": {"b3": t3 / 8.0, "b3p": t3 / 4.0},
        "t4": {"b4": 0.5},
        "b4p": {"b4p": 1.0},
        "W0": {"b4": 0.5, "b4p": (f.b4p / t4) if t4 != 0.0 else 0.0},
    }


def coupling_gradient(state):
    """dE_bind/dtheta for every name in PARAMS (and W0) on a converged
    state."""
    f = state["forces"]
    gb = b_gradient(state)
    jac = _db_dtheta(f)
    grad = {}
    for name, row in jac.items():
        grad[name] = float(sum(gb[b] * v for b, v in row.items()))
    grad["power"] = gb["power"]
    ep = state["pairs"].out[1].double().cpu().numpy()
    for q, name in ((0, "v0neut"), (1, "v0prot")):
        v0 = getattr(f, name)
        grad[name] = float(-ep[q] / v0) if (f.ipair != 0 and v0 != 0.0) else 0.0
    return grad


def force_overrides(case, theta):
    """A copy of ``case`` whose force block carries the couplings of
    ``theta`` (dict name -> value; names from PARAMS, or W0, which scales
    b4p with t4)."""
    from .forces import FORCE_TABLE
    c = copy.deepcopy(case)
    fb = c["force"]
    base = FORCE_TABLE[fb.get("name", "SLy4")]
    ov = dict(fb.get("overrides") or {})
    for k, v in theta.items():
        if k == "W0":
            t4 = ov.get("t4", base["t4"])
            b4p = ov.get("b4p", base["b4p"])
            ov["b4p"] = b4p * (v / t4) if t4 != 0.0 else b4p
            ov["t4"] = v
        elif k in ("v0neut", "v0prot"):
            fb[k] = float(v)
        else:
            ov[k] = float(v)
    fb["overrides"] = ov
    return c


def theta_of(forces):
    """Current values of PARAMS for a Forces object."""
    t = {k: getattr(forces, k) for k in PARAMS}
    t["W0"] = forces.t4
    return t


def converge(case, tol=1e-10, maxiter=3000, min_iter=30, dtype=torch.complex128, init_psi=None):
    """Self-consistent solve of ``case`` (a config case dict) until the
    binding energy changes by less than ``tol`` MeV over three successive
    iterations.  ``init_psi`` (optional) replaces the oscillator start, e.g.
    by the converged states of a nearby parameter set.  Returns (state,
    energies list)."""
    st = config.setup(case, dtype=dtype)
    if init_psi is not None:
        st["levels"].psi.copy_(init_psi)
    S = {k: st[k] for k in static._STATE_KEYS}
    static.prepare(**S)
    E, quiet = [], 0
    for i in range(1, maxiter + 1):
        static.iterate(i, **S)
        E.append(st["energies"].ehf)
        if i > 1 and abs(E[-1] - E[-2]) < tol:
            quiet += 1
        else:
            quiet = 0
        if i >= min_iter and quiet >= 3:
            break
    return st, E


def fd_gradient(case, names, rel_step=1e-4, base=None, **kw):
    """Central finite differences of the converged binding energy with a
    relative step ``rel_step`` in each coupling of ``names``.  The displaced
    solves start from the converged states of ``base`` (a converged state
    of ``case``; solved here when omitted)."""
    st0 = base if base is not None else converge(case, **kw)[0]
    th0 = theta_of(st0["forces"])
    psi0 = st0["levels"].psi
    out = {}
    for name in names:
        h = rel_step * abs(th0[name])
        ep = converge(force_overrides(case, {name: th0[name] + h}), init_psi=psi0, **kw)[0]["energies"].ehf
        em = converge(force_overrides(case, {name: th0[name] - h}), init_psi=psi0, **kw)[0]["energies"].ehf
        out[name] = (ep - em) / (2.0 * h)
    return out


class BindingEnergy(torch.autograd.Function):
    """E_bind(theta) for a vector of couplings (order ``names``): the forward
    pass converges the case at theta, the backward pass returns the explicit
    gradient at that fixed point."""

    @staticmethod
    def forward(ctx, theta, case, names, tol):
        vals = {n: float(v) for n, v in zip(names, theta.detach().cpu().tolist())}
        st, _ = converge(force_overrides(case, vals), tol=tol)
        g = coupling_gradient(st)
        ctx.save_for_backward(torch.tensor([g[n] for n in names], dtype=theta.dtype, device=theta.device))
        return torch.tensor(st["energies"].ehf, dtype=theta.dtype, device=theta.device)

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        return grad_out * g, None, None, None


def binding_energy(theta, case, names, tol=1e-10):
    """Differentiable E_bind(theta); see BindingEnergy."""
    return BindingEnergy.apply(theta, case, tuple(names), tol)


# ---------------------------------------------------------------------------
# Implicit adjoint for observables that are not variational: the proton
# point rms radius.
#
# At the fixed point the occupied states satisfy g_i = q h[rho] psi_i = 0
# (q = 1 - sum_occ |psi_j><psi_j| over the occupied states of the same
# isospin as psi_i; in the converged BCS basis h psi_i =
# e_i psi_i).  A change of theta moves them by dpsi = -H2^-1 dg/dtheta, with
# H2 the occupied-virtual block of the orbital Hessian,
#     (H2 v)_i = q (h - e_i) v_i + q dh[v] psi_i,
# dh[v] the mean field induced by the density change of v (all Skyrme
# densities and the Coulomb potential), here the central difference of the
# densities -> potentials map on the device.  The radius responds as
# dr = 2 <f psi, dpsi> with f = (|x - R_p|^2 - r^2) / (2 Z r) on the proton
# states, so with z = H2^-1 q f psi (the adjoint solve: preconditioned
# conjugate gradients with the (E0 + T)^-1 kernel of the gradient step),
#     dr/dtheta_p = -2 <z, q (dh/dtheta_p) psi>,
# dh/dtheta_p the change of the mean field with the coupling at fixed
# densities (central difference in theta_p).  <a, b> = wxyz Re sum_i
# <a_i|b_i> throughout.  The occupations are held fixed: exact for integer
# occupations (closed shells, collapsed pairing such as Ca48); with active
# pairing the response of the BCS occupations is not included (rms_gradient
# refuses fractional occupations unless told otherwise).
# ---------------------------------------------------------------------------
import types as _types


def _states_like(n, grids, dtype=torch.complex128):
    return torch.zeros((n, 2, grids.nx, grids.ny, grids.nz), dtype=dtype, device="cuda")


class RmsResponse:
    """Linear response of the proton rms radius at a converged FP64 state."""

    def __init__(self, state, fd_rel=1e-5, allow_fractional=False):
        from .densities import init_densities
        from .meanfield import init_meanfield
        from .coulomb import init_coulomb
        from .output import calculate_complete_observables
        st = state
        self.st = st
        self.g = g = st["grids"]
        lv = st["levels"]
        if lv.psi.dtype != torch.complex128:
            raise TypeError("the response solve runs on FP64 states")
        w = (lv.wocc * lv.wstates).detach().cpu().numpy()
        frac = float(np.max(np.minimum(np.abs(w), np.abs(1.0 - w))))
        if frac > 1e-6 and not allow_fractional:
            raise ValueError(f"fractional occupations (max distance from 0/1: {frac:.2e}): the BCS response is not "
                             "included; pass allow_fractional=True to hold them fixed")
        occ = np.where(w > 0.5)[0]
        self.nocc = len(occ)
        self.nn = int(np.sum(occ < lv.npsi[0]))
        idx = torch.tensor(occ, dtype=torch.long, device="cuda")
        self.psi = lv.psi.index_select(0, idx).contiguous()
        self.eps = lv.sp_energy.index_select(0, idx).contiguous()
        self.neg_eps = (-self.eps).contiguous()
        self.fd_rel = fd_rel
        self.mf0 = st["meanfield"]
        self.mf0.pack(torch.complex128)
        self.ones = torch.ones(self.nocc, dtype=torch.float64, device="cuda")
        self.zeros = torch.zeros(self.nocc, dtype=torch.float64, device="cuda")
        self.dens = [init_densities(g) for _ in range(2)]
        self.mf = [init_meanfield(g) for _ in range(2)]
        self.coul = [init_coulomb(g) for _ in range(2)]
        self.tmp = _states_like(self.nocc, g)
        self.y = [_states_like(self.nocc, g) for _ in range(2)]
        self.scal = torch.zeros(4, dtype=torch.float64, device="cuda")
        obs = calculate_complete_observables(st["densities"], lv, g)
        self.rms = float(obs.rms[1])
        self.npro = float(obs.pnr[1])
        cm = (C.c_double * 3)(*[float(v) for v in obs.cm[:, 1]])
        self.field = torch.empty((g.nx, g.ny, g.nz), dtype=torch.float64, device="cuda")
        call("hfb_rms_field", g.ctx.handle, cm, self.rms, 1.0 / (2.0 * self.npro * self.rms), ptr(self.field),
             stream_ptr())

    # ---- state algebra on the device
    def dot(self, a, b):
        call("hfb_state_dot", self.g.ctx.handle, HFB_F64, self.nocc, ptr(a), ptr(b), ptr(self.scal), stream_ptr())
        return float(self.scal[0])

    def axpby(self, a, x, b, y):
        call("hfb_state_axpby", self.g.ctx.handle, HFB_F64, self.nocc, float(a), ptr(x), float(b), ptr(y),
             stream_ptr())

    def project(self, v):
        """v_j -= sum_i <psi_i|v_j> psi_i within each isospin: orthonormality
        holds per isospin only, and neutron and proton orbitals of the same
        shape overlap almost fully, so a projection over all occupied
        states at once is not a projector."""
        for lo, hi in ((0, self.nn), (self.nn, self.nocc)):
            if hi > lo:
                call("hfb_state_project", self.g.ctx.handle, HFB_F64, hi - lo, ptr(self.psi[lo:hi]), hi - lo,
                     ptr(v[lo:hi]), stream_ptr())

    def hpsi(self, pot, x, out):
        call("hfb_hpsi", self.g.ctx.handle, HFB_F64, ptr(pot), self.nocc, self.nn, ptr(x), ptr(self.ones),
             ptr(self.zeros), ptr(out), None, None, stream_ptr())

    def _mean_field(self, k, psi, forces=None, densities=None):
        """Potentials (packed, FP64) from the densities of ``psi`` (occupied,
        weight 1) or from ``densities``, into scratch slot k."""
        from .densities import add_density
        from .meanfield import skyrme
        st = self.st
        d = densities
        if d is None:
            d = self.dens[k]
            lv = _types.SimpleNamespace(psi=psi, nstmax=self.nocc, npsi=[self.nn, self.nocc - self.nn],
                                        wocc=self.ones, wguv=self.zeros, pairwg=self.ones, wstates=self.ones)
            add_density(d, self.g, lv)
        skyrme(self.coul[k], d, forces if forces is not None else st["forces"], self.g, self.mf[k], st["params"],
               st["static"], dtype=torch.complex128)
        return self.mf[k].pot

    def induced(self, v, out):
        """out = dh[v] psi (central difference of the densities -> mean field map)."""
        nv = math.sqrt(max(self.dot(v, v), 1e-300))
        e = self.fd_rel * math.sqrt(self.nocc) / nv
        for k, sgn in ((0, 1.0), (1, -1.0)):
            self.tmp.copy_(self.psi)
            self.axpby(sgn * e, v, 1.0, self.tmp)
            pot = self._mean_field(k, self.tmp)
            self.hpsi(pot, self.psi, self.y[k])
        out.copy_(self.y[0])
        self.axpby(-1.0, self.y[1], 1.0, out)
        self.axpby(0.0, out, 1.0 / (2.0 * e), out)

    def hessian(self, v, out):
        """out = H2 v for v in the virtual space."""
        self.induced(v, out)
        self.hpsi(self.mf0.pot, v, self.y[0])
        call("hfb_state_axpby_diag", self.g.ctx.handle, HFB_F64, self.nocc, ptr(self.neg_eps), ptr(v), 1.0,
             ptr(self.y[0]), stream_ptr())
        self.axpby(1.0, self.y[0], 1.0, out)
        self.project(out)

    def precondition(self, r, out):
        """out = q (E0 + T)^-1 r (the gradient step's preconditioner)."""
        from .levels import laplace
        st = self.st
        out.copy_(laplace(None, 0, self.g, st["forces"], None, 1.0, 0.0, r, 0.0, st["static"].e0dmp))
        self.project(out)

    def rhs(self, out):
        """q f psi on the proton states (neutron part zero)."""
        out.zero_()
        npro = self.nocc - self.nn
        if npro > 0:
            call("hfb_state_mul_field", self.g.ctx.handle, HFB_F64, npro, ptr(self.field), ptr(self.psi[self.nn:]),
                 ptr(out[self.nn:]), stream_ptr())
        self.project(out)

    def solve(self, b, tol=1e-9, maxiter=500):
        """Preconditioned conjugate gradients for H2 x = b; returns (x,
        iterations, relative residual)."""
        g = self.g
        x = _states_like(self.nocc, g)
        r = b.clone()
        z = _states_like(self.nocc, g)
        self.precondition(r, z)
        p = z.clone()
        ap = _states_like(self.nocc, g)
        rz = self.dot(r, z)
        bn = math.sqrt(self.dot(b, b))
        it, res = 0, 1.0
        for it in range(1, maxiter + 1):
            self.hessian(p, ap)
            alpha = rz / self.dot(p, ap)
            self.axpby(alpha, p, 1.0, x)
            self.axpby(-alpha, ap, 1.0, r)
            res = math.sqrt(self.dot(r, r)) / bn
            if res < tol:
                break
            self.precondition(r, z)
            rz_new = self.dot(r, z)
            self.axpby(1.0, z, rz_new / rz, p)
            rz = rz_new
        return x, it, res

    def dg_dtheta(self, name, out, rel_step=1e-4):
        """out = q (dh/dtheta) psi at fixed densities (central difference)."""
        st = self.st
        th = theta_of(st["forces"])
        h = rel_step * abs(th[name]) if th[name] != 0.0 else rel_step
        for k, sgn in ((0, 1.0), (1, -1.0)):
            f = _forces_at(st["forces"], name, th[name] + sgn * h)
            pot = self._mean_field(k, None, forces=f, densities=st["densities"])
            self.hpsi(pot, self.psi, self.y[k])
        out.copy_(self.y[0])
        self.axpby(-1.0, self.y[1], 1.0, out)
        self.axpby(0.0, out, 1.0 / (2.0 * h), out)
        self.project(out)


def _forces_at(forces, name, value):
    """A copy of ``forces`` with one coupling changed and the derived
    coefficients recomputed (h2m keeps the state's (A-1)/A scaling)."""
    f = copy.copy(forces)
    f.h2m = list(forces.h2m)
    if name == "W0":
        if forces.t4 != 0.0:
            f.b4p = forces.b4p * (value / forces.t4)
        f.t4 = value
    else:
        setattr(f, name, float(value))
    return f.derive()


def rms_gradient(state, names=PARAMS, tol=1e-9, maxiter=500, allow_fractional=False):
    """d r_rms(protons) / d theta for the couplings ``names`` at a converged
    FP64 state by the implicit adjoint (see RmsResponse).  Returns (dict,
    info) with info = CG iterations and final relative residual."""
    resp = RmsResponse(state, allow_fractional=allow_fractional)
    b = _states_like(resp.nocc, resp.g)
    resp.rhs(b)
    z, it, res = resp.solve(b, tol=tol, maxiter=maxiter)
    dg = _states_like(resp.nocc, resp.g)
    out = {}
    for name in names:
        resp.dg_dtheta(name, dg)
        out[name] = -2.0 * resp.dot(z, dg)
    return out, dict(cg_iterations=it, residual=res, rms=resp.rms, occupied=resp.nocc)


def converge_states(case, tol_r=1e-13, maxiter=4000, min_iter=60, dtype=torch.complex128, init_psi=None):
    """Self-consistent solve until the proton rms radius changes by less
    than ``tol_r`` fm over three successive iterations (the states, not only
    the variational energy, converged).  Returns (state, r history)."""
    from .output import rms_radii
    st = config.setup(case, dtype=dtype)
    if init_psi is not None:
        st["levels"].psi.copy_(init_psi)
    S = {k: st[k] for k in static._STATE_KEYS}
    static.prepare(**S)
    R, quiet = [], 0
    for i in range(1, maxiter + 1):
        static.iterate(i, **S)
        R.append(rms_radii(st["densities"], st["grids"])[1][1])
        quiet = quiet + 1 if (i > 1 and abs(R[-1] - R[-2]) < tol_r) else 0
        if i >= min_iter and quiet >= 3:
            break
    return st, R


def fd_rms_gradient(case, names, rel_step=1e-4, base=None, **kw):
    """Central finite differences of the converged proton rms radius."""
    from .output import rms_radii
    st0 = base if base is not None else converge_states(case, **kw)[0]
    th0 = theta_of(st0["forces"])
    psi0 = st0["levels"].psi
    out = {}
    for name in names:
        h = rel_step * abs(th0[name])
        rp = rms_radii(*(lambda s: (s["densities"], s["grids"]))(
            converge_states(force_overrides(case, {name: th0[name] + h}), init_psi=psi0, **kw)[0]))[1][1]
        rm = rms_radii(*(lambda s: (s["densities"], s["grids"]))(
            converge_states(force_overrides(case, {name: th0[name] - h}), init_psi=psi0, **kw)[0]))[1][1]
        out[name] = (rp - rm) / (2.0 * h)
    return out


def check(case_name="Ca48", rms=True, names=SKYRME, rel_step=1e-4):
    """The sensitivities of ``case_name`` against central differences of
    the reconverged solution: {"E": {name: (gradient, fd, rel diff)},
    "rms": {...}, "cg": {...}}.  The radius part needs integer-like
    occupations (see RmsResponse); it is skipped with ``rms=False``."""
    case = config.case_dict(case_name)
    st, _ = converge(case, tol=1e-11, maxiter=3000)
    g = coupling_gradient(st)
    fd = fd_gradient(case, list(names), rel_step=rel_step, base=st, tol=1e-11, maxiter=3000)
    out = {"E": {n: (g[n], fd[n], abs(g[n] - fd[n]) / abs(fd[n])) for n in names}}
    if rms:
        sr, _ = converge_states(case, tol_r=1e-13)
        gr, info = rms_gradient(sr, list(names), tol=1e-9, allow_fractional=True)
        fr = fd_rms_gradient(case, list(names), rel_step=rel_step, base=sr, tol_r=1e-13)
        out["rms"] = {n: (gr[n], fr[n], abs(gr[n] - fr[n]) / abs(fr[n])) for n in names}
        out["cg"] = {"iterations": int(info["cg_iterations"]), "residual": float(info["residual"])}
    return out


def main(argv=None):
    """python -m hfb.adjoint [--case Ca48] [--no-rms]: print the check table
    (gradient, central difference, relative difference per coupling)."""
    import argparse
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--case", default="Ca48")
    ap.add_argument("--no-rms", action="store_true")
    args = ap.parse_args(argv)
    res = check(args.case, rms=not args.no_rms)
    for part in ("E", "rms"):
        if part not in res:
            continue
        print(f"d{'E_bind' if part == 'E' else 'r_rms(p)'}/dtheta, {args.case}:")
        for n, (a, b, r) in res[part].items():
            print(f"  {n:6s} {a:+.6e} {b:+.6e} {r:.2e}")
        print(f"  max relative difference {max(v[2] for v in res[part].values()):.2e}")
    if "cg" in res:
        print(f"  adjoint CG: {res['cg']['iterations']} iterations, residual {res['cg']['residual']:.1e}")


if __name__ == "__main__":
    main()
