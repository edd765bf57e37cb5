"""Quadrupole / principal-axis constraints (oracle; test infrastructure).

Restates constraint.py:47-342 of the reference with arrays in this
library's layout: constraint fields [nc][n][n][n] (the same field acts on
both isospins; the reference stores two identical copies in its last axis),
densities [2][n][n][n], states [nst][2][n][n][n].
"""
import numpy as np

# field kinds in the order the reference stacks them (constraint.py:126-184)
Q20, Q22, PRINCIPAL = 1, 2, 4


def constraint_fields(grids, kinds, mass_number, r0rms=0.93, damprad=6.0, dampgamma=1.0):
    """constraint.py:107-191: masked quadrupole / principal-axis fields.
    Returns (fields [nc][n][n][n], goals-order list of names)."""
    x = grids.x[:, None, None]
    y = grids.y[None, :, None]
    z = grids.z[None, None, :]
    r = np.sqrt(x ** 2 + y ** 2 + z ** 2)
    mask = 1.0 / (1.0 + np.exp((r - damprad) / dampgamma))
    norm = r0rms ** 2 * mass_number ** (5.0 / 3.0)
    out, names = [], []
    if kinds & Q20:
        out.append(np.sqrt(np.pi / 5.0) / norm * (2.0 * z ** 2 - x ** 2 - y ** 2) * mask)
        names.append("q20")
    if kinds & Q22:
        out.append(np.sqrt(1.2 * np.pi) / norm * (x ** 2 - y ** 2) * mask)
        names.append("q22")
    if kinds & PRINCIPAL:
        f = 0.5 * np.sqrt(np.pi / 5.0) / norm
        one = np.ones_like(r)
        for name, g in (("xy", x * y), ("xz", x * z), ("yz", y * z), ("x", x * one), ("y", y * one),
                        ("z", z * one)):
            out.append(f * g * mask)
            names.append(name)
    return np.stack(out), names


def expectation_values(fields, rho, wxyz):
    """constraint.py:212-245: <Q_i> = dV sum rho Q_i and the variances
    |<Q_i^2> - <Q_i>^2 / N| with N the total particle number."""
    rtot = rho[0] + rho[1]
    npart = wxyz * np.sum(rho)
    ex = wxyz * np.array([np.sum(f * rtot) for f in fields])
    m2 = wxyz * np.array([np.sum(f ** 2 * rtot) for f in fields])
    return ex, np.abs(m2 - ex ** 2 / npart)


def update_multipliers(lam, old, goals, ex, var, e0act, x0act, qeps=0.3, c0=0.8, d0=1e-4):
    """constraint.py:248-278: new multipliers and the correction factors."""
    lam_new = lam - qeps * (max(e0act, 1.0) / x0act) * (ex - old) / (2.0 * var + d0)
    qcorr = c0 * (ex - goals) / (2.0 * var + d0)
    return lam_new, qcorr


def correct_states(psi, fields, qcorr, isospin, wocc, wstates):
    """constraint.py:281-314: psi_s *= exp(wstates_s wocc_s (-sum_i qcorr_i
    Q_i)) on both spin components (isospin 0 / 1 per state)."""
    corr = -np.tensordot(qcorr, fields, axes=1)
    out = psi.copy()
    for s in range(psi.shape[0]):
        out[s] = psi[s] * np.exp(wstates[s] * wocc[s] * corr)[None]
    return out


def constraint_potential(upot, fields, lam):
    """constraint.py:196-209: upot_q -= sum_i lambda_i Q_i for both isospins."""
    return upot - np.tensordot(lam, fields, axes=1)[None]
