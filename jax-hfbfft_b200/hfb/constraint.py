"""Quadrupole / principal-axis constraints (mirror of constraint.py:47-342),
on the device, and wired into the iteration.

The reference defines the constraint module but neither its driver nor
``skyrme`` (meanfield.py:246-248) calls it.  Here a ``Constraints`` object
set on ``static.constraints`` takes part in every iteration:
``hfb.static.prepare`` measures the starting moments and adds the
constraint potential; ``hfb.static.iterate`` records the old moments before
the gradient step (before_constraint_step), after the densities updates the
multipliers and corrects the states (tune_constraints, e0act = E0 damping,
x0act = the step size) and adds the potential after ``skyrme``.  Fields,
moments, potential and correction are CUDA kernels (hfb_constraint_*); the
multiplier update is eight numbers on the host, as in the reference.
"""
import ctypes as C
import dataclasses
from dataclasses import dataclass
from typing import Any, Dict, Optional

import numpy as np
import torch

from ._lib import call, ptr, stream_ptr, prec_of

HFB_CON_Q20, HFB_CON_Q22, HFB_CON_PRINCIPAL, HFB_CON_MAX = 1, 2, 4, 8


@dataclass
class Constraints:
    """constraint.py:7-46; ``constr_field`` is a device tensor [nc, n, n, n]
    (the same field for both isospins), the crank arrays are host arrays."""
    tconstraint: bool = False
    tq_prin_axes: bool = False
    alpha20_wanted: float = -1e99
    alpha22_wanted: float = -1e99
    c0constr: float = 0.8
    d0constr: float = 1e-4
    qepsconstr: float = 0.3
    dampgamma: float = 1.0
    damprad: float = 6.0
    r0rms: float = 0.93
    numconstraint: int = 0
    constr_field: Optional[torch.Tensor] = None
    lambda_crank: Optional[np.ndarray] = None
    dlambda_crank: Optional[np.ndarray] = None
    goal_crank: Optional[np.ndarray] = None
    actual_crank: Optional[np.ndarray] = None
    old_crank: Optional[np.ndarray] = None
    actual_crank2: Optional[np.ndarray] = None
    qcorr: Optional[np.ndarray] = None

    def replace(self, **kwargs):
        return dataclasses.replace(self, **kwargs)


def _dbl(v):
    v = np.asarray(v, dtype=np.float64)
    return (C.c_double * len(v))(*v.tolist())


def init_constraints(params: Dict[str, Any], mass_number: int, grids) -> Constraints:
    """constraint.py:47-104: read alpha20_wanted / alpha22_wanted /
    tq_prin_axes and the algorithm parameters from ``params`` and build the
    fields on the device."""
    cs = Constraints()
    for k in ("alpha20_wanted", "alpha22_wanted"):
        if k in params and params[k] > -1e90:
            cs = cs.replace(**{k: float(params[k])})
    if "tq_prin_axes" in params:
        cs = cs.replace(tq_prin_axes=bool(params["tq_prin_axes"]))
    for k in ("c0constr", "d0constr", "qepsconstr", "dampgamma", "damprad", "r0rms"):
        if k in params:
            cs = cs.replace(**{k: float(params[k])})
    kinds, goals = 0, []
    if cs.alpha20_wanted > -1e90:
        kinds |= HFB_CON_Q20
        goals.append(cs.alpha20_wanted)
    if cs.alpha22_wanted > -1e90:
        kinds |= HFB_CON_Q22
        goals.append(cs.alpha22_wanted)
    if cs.tq_prin_axes:
        kinds |= HFB_CON_PRINCIPAL
        goals += [0.0] * 6
    nc = len(goals)
    if nc == 0:
        return cs
    n = grids.nx
    fields = torch.empty((nc, n, n, n), dtype=torch.float64, device="cuda")
    call("hfb_constraint_fields", grids.ctx.handle, kinds, float(mass_number), cs.r0rms, cs.damprad, cs.dampgamma,
         ptr(fields), stream_ptr())
    z = np.zeros(nc)
    return cs.replace(tconstraint=True, numconstraint=nc, constr_field=fields, lambda_crank=np.full(nc, -0.2),
                      dlambda_crank=z.copy(), goal_crank=np.array(goals), actual_crank=z.copy(), old_crank=z.copy(),
                      actual_crank2=z.copy(), qcorr=z.copy())


def add_constraint_potential(meanfield, constraints: Constraints, grids):
    """constraint.py:194-209 on the device: upot_q -= sum_i lambda_i Q_i,
    also on the packed hpsi potentials of ``meanfield``."""
    if not constraints.tconstraint or constraints.constr_field is None:
        return meanfield
    prec = 0 if meanfield.pot.dtype == torch.float64 else 1
    call("hfb_constraint_potential", grids.ctx.handle, prec, constraints.numconstraint, ptr(constraints.constr_field),
         _dbl(constraints.lambda_crank), ptr(meanfield.upot), ptr(meanfield.pot), stream_ptr())
    return meanfield


def calculate_constraint_expectation_values(densities, constraints: Constraints, grids):
    """constraint.py:212-245: expectation values and variances (host
    arrays)."""
    if not constraints.tconstraint or constraints.constr_field is None:
        return np.array([]), np.array([])
    nc = constraints.numconstraint
    out = torch.empty(2 * nc + 1, dtype=torch.float64, device="cuda")
    call("hfb_constraint_moments", grids.ctx.handle, nc, ptr(constraints.constr_field), ptr(densities.rho), ptr(out),
         stream_ptr())
    v = out.cpu().numpy()
    return v[:nc].copy(), v[nc:2 * nc].copy()


def update_lagrange_multipliers(constraints: Constraints, expectations, variances, e0act, x0act) -> Constraints:
    """constraint.py:248-278: multiplier step and correction factors."""
    if not constraints.tconstraint:
        return constraints
    den = 2.0 * variances + constraints.d0constr
    corr = -constraints.qepsconstr * (max(e0act, 1.0) / x0act) * (expectations - constraints.old_crank) / den
    return constraints.replace(lambda_crank=constraints.lambda_crank + corr,
                               qcorr=constraints.c0constr * (expectations - constraints.goal_crank) / den,
                               actual_crank=np.asarray(expectations), actual_crank2=np.asarray(variances))


def apply_wavefunction_corrections(levels, constraints: Constraints, grids):
    """constraint.py:281-314 in place on ``levels.psi``: psi_s *=
    exp(wstates_s wocc_s (-sum_i qcorr_i Q_i)) on both spin components."""
    if not constraints.tconstraint or constraints.constr_field is None:
        return levels.psi
    call("hfb_constraint_correct", grids.ctx.handle, prec_of(levels.psi), levels.nstmax, constraints.numconstraint,
         ptr(constraints.constr_field), _dbl(constraints.qcorr), ptr(levels.wocc), ptr(levels.wstates),
         ptr(levels.psi), stream_ptr())
    return levels.psi


def before_constraint_step(constraints: Constraints, densities=None) -> Constraints:
    """constraint.py:317-321."""
    if not constraints.tconstraint:
        return constraints
    return constraints.replace(old_crank=np.array(constraints.actual_crank))


def tune_constraints(constraints: Constraints, densities, levels, grids, e0act, x0act, apply_corrections=True):
    """constraint.py:324-351 (without the printout): moments, multiplier
    update and (optionally) the state correction."""
    if not constraints.tconstraint:
        return constraints, levels.psi
    ex, var = calculate_constraint_expectation_values(densities, constraints, grids)
    cs = update_lagrange_multipliers(constraints, ex, var, e0act, x0act)
    psi = apply_wavefunction_corrections(levels, cs, grids) if apply_corrections else levels.psi
    return cs, psi


def check_constraint_convergence(constraints: Constraints, tolerance: float = 0.01) -> bool:
    """constraint.py:394-404."""
    if not constraints.tconstraint:
        return True
    for a, g in zip(constraints.actual_crank, constraints.goal_crank):
        if abs(a - g) > max(tolerance, abs(g) * 0.01):
            return False
    return True


def get_constraint_summary(constraints: Constraints) -> Dict[str, Any]:
    """constraint.py:407-430."""
    if not constraints.tconstraint:
        return {"enabled": False}
    out = {"enabled": True, "numconstraint": constraints.numconstraint,
           "converged": check_constraint_convergence(constraints)}
    i = 0
    for name, want in (("Q20", constraints.alpha20_wanted), ("Q22", constraints.alpha22_wanted)):
        if want > -1e90:
            out[name] = {"target": float(constraints.goal_crank[i]), "actual": float(constraints.actual_crank[i]),
                         "lambda": float(constraints.lambda_crank[i])}
            i += 1
    if constraints.tq_prin_axes:
        out["principal_axes"] = True
    return out
