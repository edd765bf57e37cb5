"""Static iteration: initial states, gradient step, diagonalisation step and
the driver loop (mirror of static.py of jax-hfbfft).

All array work runs in libhfb on the device; the host keeps the reference's
control flow (static.py:1666-1882) and reads a handful of scalars once per
iteration (E_bind, the fluctuation measures) for the convergence test and
the step-size adaptation.
"""
from dataclasses import dataclass, field
import math
import time

import torch

from . import _lib
from ._lib import call, ptr, stream_ptr, prec_of, GrstepArgs, DiagArgs, NaturalArgs
from .densities import add_density
from .meanfield import skyrme
from .pairs import pair
from .energies import integ_energy, sum_energy
from .inout import sp_properties


@dataclass
class Static:
    tdiag: bool = False
    tlarge: bool = False
    tvaryx_0: bool = False
    ttime: bool = False
    tsort: bool = False
    maxiter: int = 40
    iternat: int = 0
    iternat_start: int = 40
    iteranneal: int = 0
    pairenhance: float = 0.0
    inibcs: int = 30
    inidiag: int = 30
    delstepbas: float = 2.0
    e0bas: float = 10.0
    outerpot: int = 0
    radinx: float = 3.1
    radiny: float = 3.1
    radinz: float = 3.1
    serr: float = 1.0e-20
    x0dmp: float = 0.45
    e0dmp: float = 100.0
    x0dmpmin: float = 0.45
    outertype: str = "N"
    hmatrix: torch.Tensor = None
    gapmatrix: torch.Tensor = None
    symcond: torch.Tensor = None
    lambda_save: torch.Tensor = None
    sums_dev: torch.Tensor = None      # running sumflu, delesum on the device
    constraints: object = None         # hfb.constraint.Constraints, or None (unconstrained)

    @property
    def sumflu(self):
        return float(self.sums_dev[0])

    @property
    def delesum(self):
        return float(self.sums_dev[1])


def init_static(forces, levels, **kwargs):
    """static.py:53-90 (also rescales h2m by (A-1)/A when zpe == 0)."""
    known = set(Static.__dataclass_fields__)
    st = Static(**{k: v for k, v in kwargs.items() if k in known})
    st.x0dmpmin = st.x0dmp
    nst = max(levels.npsi)
    for k in ("hmatrix", "gapmatrix", "symcond", "lambda_save"):
        setattr(st, k, torch.zeros((2, nst, nst), dtype=torch.complex128, device="cuda"))
    st.sums_dev = torch.zeros(4, dtype=torch.float64, device="cuda")
    if forces.zpe == 0:
        a = levels.mass_number
        forces.h2m = [h * (a - 1.0) / a for h in forces.h2m]
    return forces, st


def ho_quantum_numbers(nps):
    """(i, j, k) of the first ``nps`` states of one isospin, two spins per
    triple, shells ka = i + j + k ordered with loops k, j, i (static.py:619-660)."""
    out = []
    for ka in range(nps + 10):
        for k in range(ka + 1):
            for j in range(ka + 1):
                for i in range(ka + 1):
                    if ka == i + j + k:
                        for _ in range(2):
                            if len(out) >= nps:
                                return out
                            out.append((i, j, k))
    return out


def harmosc(grids, levels, params, static):
    """Gaussian x monomial initial states (static.py:580-738), built on the
    device; occupations reset to the first N / Z states of each isospin."""
    qn = []
    for iq in range(2):
        tr = ho_quantum_numbers(levels.npsi[iq])
        for off in range(levels.npsi[iq]):
            i, j, k = tr[off]
            qn.append((i, j, k, off % 2))
    qd = torch.tensor(qn, dtype=torch.int32, device="cuda").contiguous()
    call("hfb_harmosc", grids.ctx.handle, prec_of(levels.psi), levels.nstmax, ptr(qd), float(static.radinx),
         float(static.radiny), float(static.radinz), ptr(levels.psi), stream_ptr())
    levels.wocc.zero_()
    levels.wocc[:levels.nneut] = 1.0
    levels.wocc[levels.npsi[0]:levels.npsi[0] + levels.nprot] = 1.0
    levels.wguv.zero_()
    return levels


def grstep(forces, grids, levels, meanfield, params, static):
    """Damped-gradient step for every state (static.py:93-259)."""
    lv = levels
    rd = torch.float64 if lv.psi.dtype == torch.complex128 else torch.float32
    if meanfield.pot.dtype != rd:
        meanfield.pack(lv.psi.dtype)
    a = GrstepArgs()
    a.nst, a.nneut = lv.nstmax, lv.npsi[0]
    a.tbcs = int(bool(forces.tbcs))
    a.use_lagrange = int(params.iteration > 1 and not forces.tbcs)
    a.do_fluct = int(params.mprint > 0 and params.iteration % params.mprint == 0)
    a.x0dmp, a.e0dmp, a.h2ma, a.wxyz = float(static.x0dmp), float(static.e0dmp), float(forces.h2ma), grids.wxyz
    a.pot, a.v_pair = ptr(meanfield.pot), ptr(meanfield.v_pair)
    a.psi, a.hampsi, a.hmfpsi, a.delpsi = ptr(lv.psi), ptr(lv.hampsi), ptr(lv.hmfpsi), ptr(lv.delpsi)
    a.lagrange = ptr(lv.lagrange)
    a.wocc, a.wguv, a.pairwg, a.wstates = ptr(lv.wocc), ptr(lv.wguv), ptr(lv.pairwg), ptr(lv.wstates)
    a.sp_energy, a.sp_efluct1, a.sp_efluct2 = ptr(lv.sp_energy), ptr(lv.sp_efluct1), ptr(lv.sp_efluct2)
    sums = static.sums_dev[2:4]
    a.sums = ptr(sums)
    x0d = getattr(static, "x0_dev", None)       # step size kept on the device (graph replays)
    a.x0dmp_dev = ptr(x0d) if x0d is not None else None
    call("hfb_grstep", grids.ctx.handle, prec_of(lv.psi), a, stream_ptr())
    static.sums_dev[0:2] += sums
    # delpsi = v_pair * psi_new (static.py:203, 250): diagstep forms it on the fly
    lv._v_pair = meanfield.v_pair
    return levels, static


def diagstep(energies, forces, grids, levels, static, diagonalize=False, construct=True, npsi_neutron=None,
             npsi_proton=None):
    """Loewdin orthonormalisation, optional diagonalisation of lambda, h and
    gap matrices in the new basis, lambda and the Lagrange fields
    (static.py:261-577)."""
    lv = levels
    a = DiagArgs()
    a.npsi[0], a.npsi[1] = lv.npsi
    a.nmax = max(lv.npsi)
    a.diagonalize, a.construct = int(bool(diagonalize)), int(bool(construct))
    a.ipair, a.tbcs = int(forces.ipair), int(bool(forces.tbcs))
    a.wxyz = grids.wxyz
    a.psi, a.psi_out = ptr(lv.psi), ptr(lv.psi_spare)
    a.hampsi, a.hmfpsi, a.lagrange = ptr(lv.hampsi), ptr(lv.hmfpsi), ptr(lv.lagrange)
    vpair = getattr(lv, "_v_pair", None)
    if vpair is None:   # before the first gradient step delpsi is zero (levels.py:69)
        vpair = torch.zeros((2, grids.nx, grids.ny, grids.nz), dtype=torch.float64, device=lv.psi.device)
    a.v_pair = ptr(vpair)
    a.wocc, a.wguv, a.pairwg, a.wstates = ptr(lv.wocc), ptr(lv.wguv), ptr(lv.pairwg), ptr(lv.wstates)
    a.sp_norm, a.sp_energy, a.deltaf = ptr(lv.sp_norm), ptr(lv.sp_energy), ptr(lv.deltaf)
    a.hmatrix, a.gapmatrix = ptr(static.hmatrix), ptr(static.gapmatrix)
    a.symcond, a.lambda_save = ptr(static.symcond), ptr(static.lambda_save)
    a.efluct = ptr(energies.efluct_dev)
    call("hfb_diagstep", grids.ctx.handle, prec_of(lv.psi), a, stream_ptr())
    lv.psi, lv.psi_spare = lv.psi_spare, lv.psi
    return energies, levels, static


def lastdiag(forces, grids, levels, params, static, pairs, isospin, reference_indexing=False):
    """Quasiparticle energies (ascending) and lower-component norms of one
    isospin after convergence (static.py:1072-1168), from the h and gap
    matrices of the last diagonalisation step, the occupations and the
    Fermi energy; returns two device tensors.  By default the isospin's
    whole block of states is used (start npmin, npsi states).  The
    reference takes the first nneut / nprot states from index 0 / nneut
    (static.py:1074-1084), which for protons is not the proton block unless
    nneut == npsi[0]; ``reference_indexing=True`` restates those ranges."""
    lv = levels
    if reference_indexing:
        nst = lv.nneut if isospin == 0 else lv.nprot
        start = 0 if isospin == 0 else lv.nneut
    else:
        nst = lv.npsi[isospin]
        start = 0 if isospin == 0 else lv.npsi[0]
    ld = static.hmatrix.shape[-1]
    if nst > ld or start + nst > lv.nstmax:
        raise ValueError(f"lastdiag: {nst} states from {start} do not fit the matrices ({ld}) / states")
    e = torch.empty(nst, dtype=torch.float64, device="cuda")
    q = torch.empty(nst, dtype=torch.float64, device="cuda")
    w = lv.wocc[start:start + nst].contiguous()
    call("hfb_lastdiag", grids.ctx.handle, nst, ld, ptr(static.hmatrix[isospin]), ptr(static.gapmatrix[isospin]),
         ptr(w), ptr(pairs.out[0, isospin:isospin + 1].contiguous()), start, ptr(e), ptr(q), stream_ptr())
    return e, q


def hfb_natural(forces, grids, levels, meanfield, params, static, isospin, iternat, pairs=None,
                reference_indexing=False):
    """Configuration-space sub-iterations (static.py:920-1070): a damped
    gradient step on a unitary transformation of the isospin's states driven
    by symcond, orthonormalised by QR, the h and gap matrices transformed;
    at the end the states and Lagrange fields are rotated and the block's
    matrices replaced.  With pairing the BCS solver runs between
    sub-iterations -- here ``pair()`` with ``pairs`` (the reference's
    single-isospin call, static.py:988, lacks an argument and its last call
    passes no pairs object; the other isospin's inputs are unchanged, so
    solving both is the same as solving one).  Block: the isospin's whole
    block (npmin, npsi) by default, the reference's ranges (first nneut /
    nprot states from 0 / nneut) with ``reference_indexing=True``.  Like the
    reference, the Lagrange fields become psi_new htran (static.py:1018)."""
    lv = levels
    if reference_indexing:
        nst = lv.nneut if isospin == 0 else lv.nprot
        start = 0 if isospin == 0 else lv.nneut
    else:
        nst = lv.npsi[isospin]
        start = 0 if isospin == 0 else lv.npsi[0]
    a = NaturalArgs()
    a.nst, a.ld, a.iq, a.start = nst, static.hmatrix.shape[-1], int(isospin), start
    a.ipair = int(forces.ipair != 0)
    a.delstepbas, a.e0bas = float(static.delstepbas), float(static.e0bas)
    a.hmatrix, a.gapmatrix = ptr(static.hmatrix), ptr(static.gapmatrix)
    a.symcond, a.lambda_save = ptr(static.symcond), ptr(static.lambda_save)
    a.sp_energy, a.deltaf = ptr(lv.sp_energy), ptr(lv.deltaf)
    a.wocc, a.wguv, a.pairwg, a.wstates = ptr(lv.wocc), ptr(lv.wguv), ptr(lv.pairwg), ptr(lv.wstates)
    h = grids.ctx.handle
    call("hfb_natural_begin", h, a, stream_ptr())
    for it in range(iternat):
        last = it == iternat - 1
        call("hfb_natural_step", h, a, int(last), stream_ptr())
        if forces.ipair != 0 and pairs is not None:
            pair(levels, meanfield, forces, params, grids, pairs)
        if not last:
            call("hfb_natural_symcond", h, a, stream_ptr())
    call("hfb_natural_end", h, prec_of(lv.psi), a, ptr(lv.psi), ptr(lv.psi_spare), ptr(lv.lagrange), stream_ptr())
    lv.psi[start:start + nst].copy_(lv.psi_spare[start:start + nst])
    return levels, static


@dataclass
class RunResult:
    history: list = field(default_factory=list)
    converged: bool = False
    iterations: int = 0
    seconds: float = 0.0


def _energies(coulomb, densities, energies, forces, grids, levels, meanfield, params, pairs):
    integ_energy(coulomb, densities, energies, forces, grids, levels, params, pairs)
    sum_energy(energies, levels, meanfield, pairs, grids=grids)
    return energies


def _active_constraints(static):
    c = getattr(static, "constraints", None)
    return c if c is not None and c.tconstraint else None


def prepare(coulomb, densities, energies, forces, grids, levels, meanfield, params, static, pairs):
    """Steps before the loop (static.py:1700-1744).  With params.trestart
    (states loaded by hfb.restart.load_state) the first diagonalisation is
    skipped and params.iteration is kept, as in static.py:1700-1704."""
    if not params.trestart:
        params.iteration = 0
        diagstep(energies, forces, grids, levels, static, False, True)
    add_density(densities, grids, levels)
    cons = _active_constraints(static)
    if cons is not None:
        from .constraint import calculate_constraint_expectation_values
        ex, var = calculate_constraint_expectation_values(densities, cons, grids)
        static.constraints = cons.replace(actual_crank=ex, actual_crank2=var)
    skyrme(coulomb, densities, forces, grids, meanfield, params, static, constraints=_active_constraints(static),
           dtype=levels.psi.dtype)
    grstep(forces, grids, levels, meanfield, params, static)
    if forces.ipair != 0:
        pair(levels, meanfield, forces, params, grids, pairs)
    diagstep(energies, forces, grids, levels, static, False, True)
    sp_properties(forces, grids, levels, None)
    _energies(coulomb, densities, energies, forces, grids, levels, meanfield, params, pairs)
    if static.tvaryx_0:
        static.x0dmp = static.x0dmp * 3.0
    static._tbcssav = forces.tbcs
    return energies


def iterate_device(i, coulomb, densities, energies, forces, grids, levels, meanfield, params, static, pairs):
    """The device work of one pass of the loop body (static.py:1755-1862):
    gradient step, diagonalisation, BCS, densities with mixing, mean field,
    energies -- no read back to the host.  Host decisions that depend on
    ``i`` (BCS / diagonalisation phases, the constant gap up to iteration
    10) are taken here, so a replay of captured iterations is only valid
    past those phases."""
    params.iteration = i
    forces.tbcs = True if i <= static.inibcs else static._tbcssav
    static.tdiag = not (i > static.inidiag)
    cons = _active_constraints(static)
    if cons is not None:
        from .constraint import before_constraint_step
        static.constraints = before_constraint_step(cons)
    grstep(forces, grids, levels, meanfield, params, static)
    if forces.tbcs:
        static.tdiag = True
    diagstep(energies, forces, grids, levels, static, static.tdiag, True)
    if forces.ipair != 0:
        pair(levels, meanfield, forces, params, grids, pairs)
    if forces.ipair != 0 and static.iternat > 0 and i > static.iternat_start and not forces.tbcs:
        # configuration-space sub-iterations (static.py:1796-1798)
        for iq in range(2):
            hfb_natural(forces, grids, levels, meanfield, params, static, iq, static.iternat, pairs=pairs)
    # densities with mixing 0.2 new + 0.8 old for rho, tau, chi, and the
    # kinetic energies of sp_properties from the same derivatives
    add_density(densities, grids, levels, mix=0.2, forces=forces)
    if cons is not None:
        # multipliers from the new densities, correction of the states
        # (constraint.py:324-351), potential added after skyrme
        from .constraint import tune_constraints
        static.constraints, _ = tune_constraints(static.constraints, densities, levels, grids, static.e0dmp,
                                                 static.x0dmp)
    skyrme(coulomb, densities, forces, grids, meanfield, params, static, constraints=_active_constraints(static),
           dtype=levels.psi.dtype)
    _energies(coulomb, densities, energies, forces, grids, levels, meanfield, params, pairs)


def iterate(i, coulomb, densities, energies, forces, grids, levels, meanfield, params, static, pairs,
            x0_schedule=None):
    """One pass of the loop body (static.py:1755-1882).  Returns True once
    efluct1 < serr.  ``x0_schedule[k]`` (optional) forces the step size of
    iteration k (the reference's adaptation compares max|lambda_asym|, which
    depends on the eigenvector basis inside degenerate subspaces)."""
    iterate_device(i, coulomb, densities, energies, forces, grids, levels, meanfield, params, static, pairs)
    energies.sync()
    grids.ctx.check(f"iteration {i}")
    en = energies
    if en.efluct1[0] < static.serr and i > 1:
        return True
    if static.tvaryx_0:
        if ((en.ehf < en.ehfprev and en.efluct1[0] < en.efluct1prev * (1.0 - 1.0e-5))
                or en.efluct2[0] < en.efluct2prev * (1.0 - 1.0e-5)):
            static.x0dmp = static.x0dmp * 1.005
        else:
            static.x0dmp = static.x0dmp * 0.8
        static.x0dmp = min(max(static.x0dmp, static.x0dmpmin), static.x0dmpmin * 5.0)
        en.efluct1prev = en.efluct1[0]
        en.efluct2prev = en.efluct2[0]
        en.ehfprev = en.ehf
    if x0_schedule is not None and i + 1 < len(x0_schedule):
        static.x0dmp = float(x0_schedule[i + 1])
    return False


def first_iteration(params):
    """First loop index: 1, or the saved iteration + 1 on a restart
    (static.py:1700-1701)."""
    return params.iteration + 1 if params.trestart else 1


def statichf(coulomb, densities, energies, forces, grids, levels, meanfield, moment, params, static, pairs,
             maxiter=None, x0_schedule=None, callback=None, de_tol=None):
    """The self-consistent loop (static.py:1666-1882, without file output).

    Stops on the reference's criterion efluct1 < serr, or, when ``de_tol`` is
    given, once |E_bind(i) - E_bind(i-1)| < de_tol.  ``callback(i, energies)``
    runs after every iteration.  Returns the reference's tuple plus a
    RunResult with the per-iteration history."""
    res = RunResult()
    t0 = time.perf_counter()
    prepare(coulomb, densities, energies, forces, grids, levels, meanfield, params, static, pairs)
    energies.sync()
    res.history.append(dict(iteration=first_iteration(params) - 1, ehf=energies.ehf, ehfint=energies.ehfint,
                            x0dmp=static.x0dmp))
    n = static.maxiter if maxiter is None else maxiter
    prev = energies.ehf
    for i in range(first_iteration(params), n + 1):
        x0_used = static.x0dmp
        done = iterate(i, coulomb, densities, energies, forces, grids, levels, meanfield, params, static, pairs,
                       x0_schedule)
        res.history.append(dict(iteration=i, ehf=energies.ehf, ehfint=energies.ehfint,
                                efluct1=energies.efluct1[0], efluct2=energies.efluct2[0], x0dmp=x0_used,
                                t=time.perf_counter() - t0))
        res.iterations = i
        if callback is not None:
            callback(i, energies)
        if de_tol is not None and abs(energies.ehf - prev) < de_tol and i > 1:
            done = True
        prev = energies.ehf
        if done:
            res.converged = True
            break
    torch.cuda.synchronize()
    res.seconds = time.perf_counter() - t0
    return (coulomb, densities, energies, forces, grids, levels, meanfield, moment, params, static, pairs), res


def to_precision(state, dtype):
    """Switch a running state dict (from hfb.config.setup) between the FP64
    (complex128) and FP32 (complex64) paths: states are converted and the
    hpsi potentials repacked; densities, matrices and energies stay FP64."""
    state["levels"].to_precision(dtype)
    state["meanfield"].pack(dtype)
    return state


def remaining_change(E, w=25):
    """Geometric estimate of E_limit - E[-1] from the last 2w+1 energies
    (ratio of successive w-iteration differences); None while the tail is
    not yet geometric.  Used by the stopping and precision-switch rules."""
    if len(E) < 2 * w + 1:
        return None
    d1 = E[-1] - E[-1 - w]
    d0 = E[-1 - w] - E[-1 - 2 * w]
    if d0 == 0.0:
        return 0.0 if d1 == 0.0 else None
    r = d1 / d0
    if not (0.0 < r < 1.0):
        return None
    return d1 * r / (1.0 - r)


_STATE_KEYS = ("coulomb", "densities", "energies", "forces", "grids", "levels", "meanfield", "params", "static",
               "pairs")


# Below this many grid points times states an FP32 iteration is not cheaper
# than an FP64 one (measured on O16, 24^3 x 20 states: 1.1 ms against 0.92
# ms; the fixed costs of the tensor-core pipelines dominate), so the mixed
# driver runs such problems in FP64 throughout.
FP32_MIN_POINTS = 1 << 20


def statichf_mixed(state, maxiter=4000, switch_mev=1e-3, floor_mev=5e-5, stop_mev=5e-5, min_tail=3,
                   on_iteration=None, fp32_min_points=FP32_MIN_POINTS):
    """Mixed-precision self-consistent loop on a state dict from
    hfb.config.setup (states complex64 at entry): FP32 bulk iterations until
    the estimated remaining energy change is below ``switch_mev`` (default
    1 keV, the bar of the time-to-converge; measured on Pb208: 6.80 s to
    within 1 keV against 6.97 s with 0.5 keV and 7.09 s with 0.2 keV, the
    converged states alike to 2e-5 MeV) (or the
    last 25 energy changes stay below the FP32 noise floor ``floor_mev``),
    then FP64 refinement until the estimated remaining change is below
    ``stop_mev``.  Problems with fewer than ``fp32_min_points`` states times
    grid points run in FP64 from the start.  ``on_iteration(i, ehf,
    precision)`` runs after each iteration.  Returns (history,
    switch_iteration)."""
    lv = state["levels"]
    if lv.psi.dtype != torch.complex128 and lv.nstmax * state["grids"].n3 < fp32_min_points:
        to_precision(state, torch.complex128)
    S = {k: state[k] for k in _STATE_KEYS}
    prepare(**S)
    S["energies"].sync()
    E = [S["energies"].ehf]
    hist = []
    switched = state["levels"].psi.dtype == torch.complex128
    switch_it = 0 if switched else None
    tail = 0
    for i in range(1, maxiter + 1):
        iterate(i, **S)
        e = S["energies"].ehf
        E.append(e)
        prec = "f64" if switched else "f32"
        hist.append((i, e, prec))
        if on_iteration is not None:
            on_iteration(i, e, prec)
        if not switched:
            rem = remaining_change(E)
            recent = [abs(E[k] - E[k - 1]) for k in range(max(1, len(E) - 25), len(E))]
            if (rem is not None and abs(rem) < switch_mev) or (len(E) > 60 and max(recent) < floor_mev):
                to_precision(state, torch.complex128)
                switched = True
                switch_it = i
                E = [e]
        else:
            tail += 1
            rem = remaining_change(E)
            if tail >= min_tail and rem is not None and abs(rem) < stop_mev:
                break
    return hist, switch_it
