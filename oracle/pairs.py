"""BCS pairing: gaps, Fermi level, occupations (oracle; test infrastructure).

Follows reference pairs.py:15-220.  The Fermi level is found with SciPy's
``brentq`` on [-100, 100] with xtol=1e-14 exactly as pairs.py:59 does.
"""
from dataclasses import dataclass, field
import numpy as np
from scipy.optimize import brentq


@dataclass
class Pairs:
    eferm: np.ndarray = field(default_factory=lambda: np.zeros(2))
    epair: np.ndarray = field(default_factory=lambda: np.zeros(2))
    avdelt: np.ndarray = field(default_factory=lambda: np.zeros(2))
    avdeltv2: np.ndarray = field(default_factory=lambda: np.zeros(2))
    avg: np.ndarray = field(default_factory=lambda: np.zeros(2))
    firstcall: bool = True


def bcs_particle_number(eferm, sp_energy, deltaf, wstates):
    """pairs.py:25-45."""
    edif = sp_energy - eferm
    eq = np.maximum(np.sqrt(edif ** 2 + deltaf ** 2), 1.0e-20)
    v2 = np.clip(0.5 * (1.0 - edif / eq), 1.0e-10, 1.0 - 1.0e-10)
    return np.sum(v2 * wstates)


def find_fermi(target, sp_energy, deltaf, wstates):
    """pairs.py:47-61."""
    return brentq(lambda e: float(bcs_particle_number(e, sp_energy, deltaf, wstates)) - target,
                  a=-100.0, b=100.0, xtol=1e-14)


def soft_cutoff(e, ecut, width):
    """pairs.py:63-64."""
    return 1.0 / (1.0 + np.exp((e - ecut) / width))


def pairdn(iq, particle_number, levels, forces, pairs):
    """One isospin of the BCS solve (pairs.py:66-131)."""
    sl = levels.block(iq)
    e = levels.sp_energy[sl]
    dlt = levels.deltaf[sl]
    ef = find_fermi(particle_number, e, dlt, levels.wstates[sl])
    pairwg = levels.pairwg.copy()
    wstates = levels.wstates.copy()
    ws_calc = levels.wstates[sl]
    if forces.pair_cutoff[iq] > 0.0:
        pairwg[sl] = soft_cutoff(e, ef + forces.pair_cutoff[iq], forces.softcut_range * forces.pair_cutoff[iq])
    if forces.state_cutoff[iq] > 0.0:
        sc = soft_cutoff(e, ef + forces.state_cutoff[iq], forces.softcut_range * forces.state_cutoff[iq])
        wstates[sl] = sc
        ws_calc = sc
    edif = e - ef
    eq = np.maximum(np.sqrt(edif ** 2 + dlt ** 2), 1.0e-20)
    v2 = 0.5 * (1.0 - edif / eq)
    uv = np.sqrt(np.maximum(v2 - v2 ** 2, 1.0e-6))
    wocc = np.clip(v2, 1e-10, 1.0 - 1e-10)
    vol = 0.5 * uv * ws_calc
    sumuv = np.sum(vol)
    sumduv = np.sum(vol * dlt)
    sumv2 = np.sum(wocc * ws_calc)
    sumdv2 = np.sum(dlt * wocc * ws_calc)
    pairs.eferm[iq] = ef
    pairs.epair[iq] = sumduv
    pairs.avdelt[iq] = sumduv / max(sumuv, 1.0e-20)
    pairs.avdeltv2[iq] = sumdv2 / max(sumv2, 1.0e-20)
    pairs.avg[iq] = sumduv / max(sumuv, 1.0e-20) ** 2
    return wocc, uv, pairwg, wstates


def pairgap(levels, mf, iteration, grids, firstcall):
    """pairs.py:133-157."""
    if iteration <= 10:
        return 11.2 / np.sqrt(levels.mass_number) * np.ones_like(levels.deltaf)
    if not firstcall:
        return levels.deltaf
    dens = np.sum((levels.psi * np.conj(levels.psi)).real, axis=1)
    vp = np.where(levels.isospin[:, None, None, None] == 0, mf.v_pair[0][None], mf.v_pair[1][None])
    return np.sum(vp * dens, axis=(1, 2, 3)) * grids.wxyz * levels.pairwg


def pair(levels, mf, forces, iteration, grids, pairs):
    """pairs.py:161-220 (printing omitted)."""
    levels.deltaf = pairgap(levels, mf, iteration, grids, pairs.firstcall)
    pairs.firstcall = False
    for iq, npart in ((0, float(levels.nneut)), (1, float(levels.nprot))):
        wocc, uv, pairwg, wstates = pairdn(iq, npart, levels, forces, pairs)
        sl = levels.block(iq)
        levels.wocc[sl] = wocc
        levels.wguv[sl] = uv
        if forces.pair_cutoff[iq] > 0.0:
            levels.pairwg = pairwg
        if forces.state_cutoff[iq] > 0.0:
            levels.wstates = wstates
    return levels, pairs
