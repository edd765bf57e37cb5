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

Parameters (``PARAMS``): t0-t3, x0-x3, W0 (= t4, with b4p scaled in
proportion, so SLy4's b4 = b4p = W0/2 move together), power (alpha), and
v0neut, v0prot.

``coupling_gradient(state)`` evaluates the gradient on a converged state;
``converge`` runs a state to a tight energy tolerance; ``fd_gradient`` is the
central finite-difference check; ``BindingEnergy`` puts the pair behind a
torch.autograd.Function (forward = self-consistent solve at theta, backward
= the explicit gradient above).
"""
import copy

import numpy as np
import torch

from . import config, static
from ._lib import call, ptr, stream_ptr

PARAMS = ("t0", "t1", "t2", "t3", "x0", "x1", "x2", "x3", "W0", "power", "v0neut", "v0prot")
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
        "W0": {"b4": 0.5, "b4p": (f.b4p / t4) if t4 != 0.0 else 0.0},
    }


def coupling_gradient(state):
    """dE_bind/dtheta for every name in PARAMS on a converged state."""
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
    ``theta`` (dict name -> value; names from PARAMS, W0 scales b4p)."""
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
    t = {k: getattr(forces, k) for k in ("t0", "t1", "t2", "t3", "x0", "x1", "x2", "x3", "power", "v0neut",
                                         "v0prot")}
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
