"""Initial states, gradient step, diagonalisation step and the iteration driver
(oracle; test infrastructure).

Follows reference static.py:21-738 and the loop body of
``statichf_with_benchmark`` (static.py:1666-1882).
"""
from dataclasses import dataclass, field
import numpy as np

from . import pool
from .spectral import laplace
from .meanfield import hpsi01, skyrme
from .densities import add_density
from .pairs import pair
from .energies import integ_energy, sum_energy, sp_properties


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
    delesum: float = 0.0
    sumflu: float = 0.0
    x0dmp: float = 0.45
    e0dmp: float = 100.0
    x0dmpmin: float = 0.45
    outertype: str = "N"
    hmatrix: np.ndarray = None
    gapmatrix: np.ndarray = None
    symcond: np.ndarray = None
    lambda_save: np.ndarray = None


def init_static(forces, levels, **kw):
    """static.py:53-90: also rescales h2m by (A-1)/A when zpe == 0."""
    nst = max(levels.npsi)
    st = Static(**kw)
    st.x0dmpmin = st.x0dmp
    for name in ("hmatrix", "gapmatrix", "symcond", "lambda_save"):
        setattr(st, name, np.zeros((2, nst, nst), dtype=np.complex128))
    if forces.zpe == 0:
        forces.h2m = forces.h2m * ((levels.mass_number - 1.0) / levels.mass_number)
    return forces, st


def rpsnorm(ps, wxyz):
    """trivial.py:5-7."""
    return wxyz * np.sum((np.conj(ps) * ps).real)


def overlap(pl, pr, wxyz):
    """trivial.py:10-12."""
    return wxyz * np.sum(np.conj(pl) * pr)


def ho_quantum_numbers(nps):
    """(i, j, k) of the first ``nps`` states of one isospin (static.py:619-660):
    shells ka = i+j+k in order, loops k, j, i outermost to innermost, two spin
    states per triple."""
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


def harmosc(grids, levels, st):
    """Gaussian x monomial initial states (static.py:580-738)."""
    x = grids.x[:, None, None]
    y = grids.y[None, :, None]
    z = grids.z[None, None, :]
    g = np.exp(-((x / st.radinx) ** 2 + (y / st.radiny) ** 2 + (z / st.radinz) ** 2))
    g = g / np.sqrt(rpsnorm(np.stack([g, np.zeros_like(g)]), grids.wxyz))
    psi = np.zeros_like(levels.psi)
    wocc = np.zeros(levels.nstmax)
    wocc[:levels.nneut] = 1.0
    wocc[levels.npsi[0]:levels.npsi[0] + levels.nprot] = 1.0
    for iq in range(2):
        sl = levels.block(iq)
        qn = ho_quantum_numbers(levels.npsi[iq])
        for off, nst in enumerate(range(sl.start, sl.stop)):
            if off == 0:
                psi[nst, 0] = g
            else:
                i, j, k = qn[off]
                poly = (grids.x ** i)[:, None, None] * (grids.y ** j)[None, :, None] * (grids.z ** k)[None, None, :]
                psi[nst, off % 2] = g * poly
            a = rpsnorm(psi[nst], grids.wxyz)
            if off == 0 or a > 1e-12:
                psi[nst] = psi[nst] / np.sqrt(a)
    levels.psi = psi
    levels.wocc = wocc
    levels.wguv = np.zeros(levels.nstmax)
    return levels


def grstep(forces, grids, levels, mf, iteration, st, mprint=1):
    """Damped-gradient step for every state (static.py:93-259)."""
    wx = grids.wxyz
    nst = levels.nstmax
    if forces.tbcs:
        wt = np.ones(nst)
        wu = np.zeros(nst)
    else:
        wt = levels.wstates * levels.wocc
        wu = levels.wstates * levels.wguv * levels.pairwg
    new_psi = np.empty_like(levels.psi)
    hampsi = np.empty_like(levels.psi)
    hmfpsi = np.empty_like(levels.psi)
    delpsi = np.empty_like(levels.psi)
    spe_new = np.zeros(nst)
    ef1 = levels.sp_efluct1.copy()
    ef2 = levels.sp_efluct2.copy()
    denerg = np.zeros(nst)
    def block(iq, sl):
        # the states of ``sl`` (all of isospin iq); writes disjoint slices
        ps1, pmf, _ = hpsi01(grids, mf, iq, wt[sl], wu[sl], levels.psi[sl])
        vmax = np.max(mf.v_pair[iq])
        for loc, k in enumerate(range(sl.start, sl.stop)):
            psin = levels.psi[k]
            p1 = ps1[loc]
            spe_new[k] = overlap(psin, pmf[loc], wx).real                      # (173)
            if st.e0dmp > 0.0:                                                 # e0dmp_gt_zero (93-146)
                hexp = overlap(psin, p1, wx).real
                if iteration > 1 and not forces.tbcs:
                    orth = p1 - levels.lagrange[k]
                else:
                    orth = p1 - hexp * psin
                if mprint > 0 and iteration % mprint == 0:
                    ef1[k] = np.sqrt(rpsnorm(orth, wx))
                    ef2[k] = np.sqrt(rpsnorm(levels.lagrange[k] - hexp * psin, wx))
                if forces.tbcs:
                    ps2 = laplace(grids, forces.h2ma, 1.0, 0.0, orth, 0.0, st.e0dmp)
                else:
                    ps2 = laplace(grids, forces.h2ma, levels.wocc[k], levels.wguv[k] * levels.pairwg[k],
                                  orth, vmax, st.e0dmp)
                new_psi[k] = psin - st.x0dmp * ps2
            else:                                                              # (181-185)
                new_psi[k] = (1.0 + st.x0dmp * (spe_new[k] - levels.sp_energy[k])) * psin - st.x0dmp * p1
            denerg[k] = (levels.sp_energy[k] - spe_new[k]) / abs(spe_new[k])
        hampsi[sl] = pmf
        _, hm, dl = hpsi01(grids, mf, iq, wt[sl], wu[sl], new_psi[sl])         # (194-208)
        hmfpsi[sl] = hm
        delpsi[sl] = dl

    jobs = []
    for iq in range(2):
        b = levels.block(iq)
        jobs += [(iq, c) for c in pool.chunks(b.start, b.stop)]
    pool.pmap(lambda j: block(*j), jobs)
    levels.psi, levels.hampsi, levels.hmfpsi, levels.delpsi = new_psi, hampsi, hmfpsi, delpsi
    levels.sp_energy = spe_new
    levels.sp_efluct1, levels.sp_efluct2 = ef1, ef2
    st.sumflu = st.sumflu + np.sum(levels.sp_efluct1)
    st.delesum = st.delesum + np.sum(levels.wocc * levels.wstates * denerg)
    return levels, st


def loewdin(psi2d, wxyz, nst):
    """S^-1/2 with an eigenvalue floor (static.py:463-482)."""
    s = (np.conj(psi2d.T) @ psi2d) * wxyz
    norm = np.diagonal(s).real.copy()
    w, v = np.linalg.eigh(s, UPLO="L")
    thr = max(1e-12, np.finfo(np.float64).eps * np.max(w) * nst)
    w = np.maximum(w, thr)
    u = v @ np.conj((v * (1.0 / np.sqrt(w))[None, :]).T)
    return u, norm


def diagstep(en, forces, grids, levels, st, diagonalize=False, construct=True):
    """Loewdin orthonormalisation, optional diagonalisation of lambda, the
    rotated h and gap matrices, lambda and the Lagrange fields
    (static.py:261-577)."""
    for iq in range(2):
        sl = levels.block(iq)
        nst = levels.npsi[iq]
        shp = levels.psi[sl].shape
        psi2d = levels.psi[sl].reshape(nst, -1).T.copy()
        u_rho, norm = loewdin(psi2d, grids.wxyz, nst)
        levels.sp_norm[sl] = norm
        if diagonalize:
            lam = (np.conj(psi2d.T) @ levels.hampsi[sl].reshape(nst, -1).T) * grids.wxyz
            _, vl = np.linalg.eigh(lam, UPLO="L")
            u = u_rho @ vl
        else:
            u = u_rho
        new2d = psi2d @ u
        levels.psi[sl] = new2d.T.reshape(shp)
        if construct:
            hm_old = (np.conj(psi2d.T) @ levels.hmfpsi[sl].reshape(nst, -1).T) * grids.wxyz
            h = np.conj(u.T) @ (hm_old @ u)
            gap = np.zeros_like(h)
            if forces.ipair != 0:
                g_old = (np.conj(psi2d.T) @ levels.delpsi[sl].reshape(nst, -1).T) * grids.wxyz
                gap = np.conj(u.T) @ (g_old @ u)
            st.hmatrix[iq, :nst, :nst] = h
            st.gapmatrix[iq, :nst, :nst] = gap
            levels.sp_energy[sl] = np.diagonal(h).real
            if forces.ipair != 0:
                levels.deltaf[sl] = np.diagonal(gap).real * levels.pairwg[sl]
            if forces.tbcs:
                st.gapmatrix[iq, :nst, :nst] = gap * np.eye(nst)
            wt = levels.wocc[sl] * levels.wstates[sl]
            wu = levels.wguv[sl] * levels.pairwg[sl] * levels.wstates[sl]
            lt = wt[None, :] * st.hmatrix[iq, :nst, :nst] - wu[None, :] * st.gapmatrix[iq, :nst, :nst]
            lasym = 0.5 * (lt - np.conj(lt.T))
            lsym = 0.5 * (lt + np.conj(lt.T))
            en.efluct1q[iq] = np.max(np.abs(lasym))
            en.efluct2q[iq] = np.sqrt(np.sum(np.abs(lasym) ** 2) / nst ** 2)
            st.symcond[iq, :nst, :nst] = lasym
            st.lambda_save[iq, :nst, :nst] = lsym
            lag = new2d @ lsym
            en.efluct1[0] = np.max(en.efluct1q)
            en.efluct2[0] = np.average(en.efluct2q)
        else:
            lag = new2d @ st.lambda_save[iq, :nst, :nst]
        levels.lagrange[sl] = lag.T.reshape(shp)
    return en, levels, st


@dataclass
class RunState:
    """Everything the driver carries between iterations."""
    params: dict
    forces: object
    grids: object
    levels: object
    mf: object
    dens: object
    coulomb: object
    st: object
    en: object
    pairs: object
    iteration: int = 0
    history: list = field(default_factory=list)


def _energies(rs):
    rs.levels = sp_properties(rs.forces, rs.grids, rs.levels)
    rs.en = integ_energy(rs.coulomb, rs.dens, rs.en, rs.forces, rs.grids, rs.levels, rs.pairs)
    rs.en = sum_energy(rs.en, rs.levels, rs.mf, rs.pairs)


def prepare(rs):
    """Pre-loop steps of the driver (static.py:1700-1744)."""
    f, g, lv = rs.forces, rs.grids, rs.levels
    mprint = rs.params.get("mprint", 1)
    rs.iteration = 0
    rs.en, lv, rs.st = diagstep(rs.en, f, g, lv, rs.st, False, True)
    rs.dens = add_density(rs.dens, g, lv)
    rs.mf, rs.coulomb = skyrme(rs.coulomb, rs.dens, f, g, rs.mf)
    lv, rs.st = grstep(f, g, lv, rs.mf, 0, rs.st, mprint)
    if f.ipair != 0:
        lv, rs.pairs = pair(lv, rs.mf, f, 0, g, rs.pairs)
    rs.en, lv, rs.st = diagstep(rs.en, f, g, lv, rs.st, False, True)
    rs.levels = lv
    _energies(rs)
    if rs.st.tvaryx_0:
        rs.st.x0dmp = rs.st.x0dmp * 3.0
    rs.tbcssav = f.tbcs
    return rs


def iterate(rs, i, x0_schedule=None):
    """One pass of the loop body (static.py:1755-1882).  Returns True once
    the efluct1 < serr criterion is met.

    ``x0_schedule[k]`` (optional) forces the step size used in iteration k.
    The reference's adaptation (static.py:1870-1878) compares efluct1 =
    max|lambda_asym|, which depends on the basis LAPACK picks inside
    degenerate subspaces; replaying a recorded schedule makes two correct
    implementations follow the same trajectory."""
    f, g, st = rs.forces, rs.grids, rs.st
    mprint = rs.params.get("mprint", 1)
    rs.iteration = i
    f.tbcs = True if i <= st.inibcs else rs.tbcssav
    st.tdiag = not (i > st.inidiag)
    lv, st = grstep(f, g, rs.levels, rs.mf, i, st, mprint)
    if f.tbcs:
        st.tdiag = True
    rs.en, lv, st = diagstep(rs.en, f, g, lv, st, st.tdiag, True)
    if f.ipair != 0:
        lv, rs.pairs = pair(lv, rs.mf, f, i, g, rs.pairs)
    if f.ipair != 0 and st.iternat > 0 and i > st.iternat_start and not f.tbcs:   # (1796-1798)
        def hook(levels):
            _, rs.pairs = pair(levels, rs.mf, f, i, g, rs.pairs)
        for iq in range(2):
            lv, st = hfb_natural(lv, st, iq, st.iternat, ipair=f.ipair, pair_hook=hook)
    old = (rs.dens.rho.copy(), rs.dens.tau.copy(), rs.dens.chi.copy())
    rs.dens = add_density(rs.dens, g, lv)
    addnew = 0.2
    rs.dens.rho = addnew * rs.dens.rho + (1.0 - addnew) * old[0]
    rs.dens.tau = addnew * rs.dens.tau + (1.0 - addnew) * old[1]
    rs.dens.chi = addnew * rs.dens.chi + (1.0 - addnew) * old[2]
    rs.mf, rs.coulomb = skyrme(rs.coulomb, rs.dens, f, g, rs.mf)
    rs.levels = lv
    _energies(rs)
    en = rs.en
    rs.history.append(dict(iteration=i, ehf=float(en.ehf), ehfint=float(en.ehfint),
                           efluct1=float(en.efluct1[0]), efluct2=float(en.efluct2[0]), x0dmp=float(st.x0dmp)))
    if en.efluct1[0] < st.serr and i > 1:
        return True
    if st.tvaryx_0:
        if ((en.ehf < en.ehfprev and en.efluct1[0] < en.efluct1prev * (1.0 - 1.0e-5))
                or en.efluct2[0] < en.efluct2prev * (1.0 - 1.0e-5)):
            st.x0dmp = st.x0dmp * 1.005
        else:
            st.x0dmp = st.x0dmp * 0.8
        st.x0dmp = float(np.clip(st.x0dmp, st.x0dmpmin, st.x0dmpmin * 5.0))
        en.efluct1prev = en.efluct1[0]
        en.efluct2prev = en.efluct2[0]
        en.ehfprev = en.ehf
    if x0_schedule is not None and i + 1 < len(x0_schedule):
        st.x0dmp = float(x0_schedule[i + 1])
    return False


def build(case):
    """Construct a ready-to-run state from a case dict with keys ``grid``,
    ``force``, ``levels``, ``static`` and ``mprint`` (the order of set-up
    follows the reference's run_hfb, test.py:145-166)."""
    from .model import init_grids, init_forces, init_levels
    from .meanfield import init_meanfield
    from .densities import init_densities
    from .coulomb import init_coulomb
    from .energies import Energies
    from .pairs import Pairs
    g = init_grids(**case["grid"])
    fk = dict(case["force"])
    f = init_forces(**fk)
    lv = init_levels(g, **case["levels"])
    f, st = init_static(f, lv, **case["static"])
    lv = harmosc(g, lv, st)
    return RunState(params=dict(mprint=case.get("mprint", 1)), forces=f, grids=g, levels=lv,
                    mf=init_meanfield(g), dens=init_densities(g), coulomb=init_coulomb(g), st=st,
                    en=Energies(), pairs=Pairs())


def run(rs, maxiter=None, callback=None):
    """Pre-loop steps then iterations until convergence or ``maxiter``."""
    prepare(rs)
    n = rs.st.maxiter if maxiter is None else maxiter
    for i in range(1, n + 1):
        done = iterate(rs, i)
        if callback is not None:
            callback(rs, i)
        if done:
            break
    return rs


def lastdiag_block(h, gap, w, eferm, first):
    """Quasiparticle energies and lower-component norms of one block
    (static.py:1072-1168).  ``h``, ``gap``: the block's (nst, nst) corners of
    the h and gap matrices; ``w``: the occupations of the block's states;
    ``first``: the index of the block's first state in the whole state array
    (the parity of a state's index picks its time-reversal partner,
    static.py:1129-1139).  Returns (energies ascending, norms)."""
    nst = h.shape[0]
    wi, wj = w[:, None], w[None, :]
    xi = -np.sqrt(wi * wj) + np.sqrt((1.0 - wi) * (1.0 - wj))                # (1105-1106)
    eta = np.sqrt(wi * (1.0 - wj)) + np.sqrt(wj * (1.0 - wi))                 # (1108-1109)
    hm = h - eferm * np.eye(nst)                                              # (1116-1117)
    m = hm * xi + gap * eta                                                   # (1120)
    e, u = np.linalg.eigh(m, UPLO="L")                                        # (1124)
    c = np.zeros((nst, nst))
    for i in range(nst):                                                      # (1129-1139)
        g = first + i
        if g % 2 == 0 and i >= 1:
            c[i, i - 1] = -np.sqrt(w[i])
        if g % 2 == 1 and i + 1 < nst:
            c[i, i + 1] = np.sqrt(w[i])
    low = c @ u
    norm = np.sqrt(np.sum(np.abs(low) ** 2, axis=0))                          # (1142-1148)
    order = np.argsort(e, kind="stable")                                      # (1151-1153)
    return e[order], norm[order]


def lastdiag(levels, st, eferm, iq, reference_indexing=False):
    """lastdiag for isospin ``iq``.  The reference takes the first nneut
    (nprot) states starting at index 0 (nneut), static.py:1074-1084: for
    protons that is not the proton block unless nneut == npsi[0], and it
    leaves out the unoccupied states of each block.  By default the whole
    block of the isospin is used (start npmin, size npsi);
    ``reference_indexing=True`` restates the reference's ranges."""
    if reference_indexing:
        nst = levels.nneut if iq == 0 else levels.nprot
        start = 0 if iq == 0 else levels.nneut
    else:
        nst = levels.npsi[iq]
        start = 0 if iq == 0 else levels.npsi[0]
    return lastdiag_block(st.hmatrix[iq, :nst, :nst], st.gapmatrix[iq, :nst, :nst],
                          np.asarray(levels.wocc)[start:start + nst], float(eferm[iq]), start)


def calc_lambda(h, gap, wt, wu):
    """Symmetric lambda of the sub-iterations (static.py:1030-1046):
    lambda_temp[:, j] = wt_j h[:, j] - wu_j gap[:, j], lambda = (lt + lt^H)/2."""
    lt = h * wt[None, :] - gap * wu[None, :]
    return 0.5 * (lt + np.conj(lt.T))


def hfb_natural(levels, st, iq, iternat, ipair=0, pair_hook=None, reference_indexing=False):
    """Configuration-space sub-iterations (static.py:920-1070): a damped
    gradient step on the unitary transformation ``cm`` driven by symcond,
    orthonormalised by QR, the h and gap matrices transformed, and at the end
    the states and Lagrange fields rotated.  With ``ipair != 0`` the
    reference calls the pairing solver between sub-iterations
    (``pair_hook(levels)``; its single-isospin call, static.py:988, has the
    wrong number of arguments, and the last one passes no pairs object).
    The block: the isospin's whole block by default; the reference's ranges
    (first nneut / nprot states from index 0 / nneut) with
    ``reference_indexing=True``.  The reference passes the transformed h
    (not lambda) to the Lagrange-field update (static.py:1018, 1048-1068);
    restated as written."""
    if reference_indexing:
        nst = levels.nneut if iq == 0 else levels.nprot
        start = 0 if iq == 0 else levels.nneut
    else:
        nst = levels.npsi[iq]
        start = 0 if iq == 0 else levels.npsi[0]
    sl = slice(start, start + nst)
    cm = np.eye(nst, dtype=np.complex128)
    spe = levels.sp_energy
    if st.e0bas == 0.0:
        dampstep = np.full(nst, st.delstepbas / (np.max(spe[sl]) - np.min(spe[sl])))
    else:
        dampstep = st.delstepbas / (spe[sl] - spe[start] + st.e0bas)
    hmat = st.hmatrix[iq, :nst, :nst].copy()
    gapmat = st.gapmatrix[iq, :nst, :nst].copy()

    def weights():
        wt = levels.wocc[sl] * levels.wstates[sl]
        wu = levels.wguv[sl] * levels.pairwg[sl] * levels.wstates[sl]
        return wt, wu

    htran = gaptran = None
    for it in range(iternat):
        cm = cm - dampstep[:, None] * st.symcond[iq, :nst, :nst]                  # (952-957)
        cm, _ = np.linalg.qr(cm)                                                   # (959-960)
        htran = np.conj(cm.T) @ hmat @ cm                                          # (964-965)
        gaptran = np.conj(cm.T) @ gapmat @ cm
        hcm = hmat @ cm                                                            # (968-969)
        gapcm = gapmat @ cm
        if ipair != 0 or it == iternat - 1:                                        # (972-992)
            levels.sp_energy[sl] = np.diag(htran).real
            if ipair != 0:
                levels.deltaf[sl] = np.diag(gaptran).real * levels.pairwg[sl]
                if pair_hook is not None:
                    pair_hook(levels)
        if it < iternat - 1:                                                       # (994-1015)
            wt, wu = weights()
            cml = cm @ calc_lambda(htran, gaptran, wt, wu)
            st.symcond[iq, :nst, :nst] = hcm * wt[None, :] - gapcm * wu[None, :] - cml
    shp = levels.psi[sl].shape
    old = levels.psi[sl].reshape(nst, -1)                                          # (1018, 1048-1068)
    new = cm.T @ old
    levels.psi[sl] = new.reshape(shp)
    levels.lagrange[sl] = (htran.T @ new).reshape(shp)
    st.hmatrix[iq, :nst, :nst] = htran                                             # (1021-1022)
    st.gapmatrix[iq, :nst, :nst] = gaptran
    wt, wu = weights()
    st.lambda_save[iq, :nst, :nst] = calc_lambda(htran, gaptran, wt, wu)           # (1025-1026)
    return levels, st
