"""Energies, single-particle properties and radii (oracle; test infrastructure).

Follows reference energies.py:8-372, inout.py:64-150 and output.py:177-246.
"""
from dataclasses import dataclass, field
import numpy as np

from . import pool
from .model import apply_along
from .spectral import cderv01, k2_total


@dataclass
class Energies:
    ehft: float = 0.0
    ehf0: float = 0.0
    ehf1: float = 0.0
    ehf2: float = 0.0
    ehf3: float = 0.0
    ehfls: float = 0.0
    ehflsodd: float = 0.0
    ehfc: float = 0.0
    ecorc: float = 0.0
    ehfint: float = 0.0
    efluct1: np.ndarray = field(default_factory=lambda: np.zeros(1))
    efluct1q: np.ndarray = field(default_factory=lambda: np.zeros(2))
    efluct1prev: float = 0.0
    efluct2: np.ndarray = field(default_factory=lambda: np.zeros(1))
    efluct2q: np.ndarray = field(default_factory=lambda: np.zeros(2))
    efluct2prev: float = 0.0
    tke: float = 0.0
    ehf: float = 0.0
    ehfprev: float = 0.0
    e3corr: float = 0.0
    e_zpe: float = 0.0
    orbital: np.ndarray = field(default_factory=lambda: np.zeros(3))
    spin: np.ndarray = field(default_factory=lambda: np.zeros(3))
    total_angmom: np.ndarray = field(default_factory=lambda: np.zeros(3))
    ehfCrho0: float = 0.0
    ehfCrho1: float = 0.0
    ehfCdrho0: float = 0.0
    ehfCdrho1: float = 0.0
    ehfCtau0: float = 0.0
    ehfCtau1: float = 0.0
    ehfCdJ0: float = 0.0
    ehfCdJ1: float = 0.0
    ehfCj0: float = 0.0
    ehfCj1: float = 0.0


def integ_energy(coulomb, dens, en, forces, grids, levels, pairs, tcoul=True):
    """EDF integrals (energies.py:90-306).  Mutates and returns ``en``."""
    f, w = forces, grids.wxyz
    D1, D2 = grids.der1, grids.der2
    rho, tau, cur, sd, so = dens.rho, dens.tau, dens.current, dens.sdens, dens.sodens
    lap = np.stack([sum(apply_along(D2[a], rho[iq], a) for a in range(3)) for iq in range(2)])
    rn, rp = rho[0], rho[1]
    rt = rn + rp
    r1 = -rn + rp
    d2 = lap[0] + lap[1]
    d21 = -lap[0] + lap[1]
    t0 = tau[0] + tau[1]
    t1 = -tau[0] + tau[1]
    en.ehf0 = w * np.sum((f.b0 * rt ** 2 - f.b0p * (rp ** 2 + rn ** 2)) / 2.0)
    en.ehfCrho0 = w * np.sum((f.Crho0 + f.Crho0D * rt ** f.power) * rt ** 2)
    en.ehfCrho1 = w * np.sum((f.Crho1 + f.Crho1D * rt ** f.power) * r1 ** 2)
    en.ehf3 = w * np.sum(rt ** f.power * (f.b3 * rt ** 2 - f.b3p * (rp ** 2 + rn ** 2)) / 3.0)
    en.ehf2 = w * np.sum((-f.b2 * rt * d2 + f.b2p * (rp * lap[1] + rn * lap[0])) / 2.0)
    en.ehfCdrho0 = w * np.sum(f.Cdrho0 * rt * d2)
    en.ehfCdrho1 = w * np.sum(f.Cdrho1 * r1 * d21)
    en.ehfCtau0 = w * np.sum(f.Ctau0 * t0 * rt)
    en.ehfCtau1 = w * np.sum(f.Ctau1 * t1 * r1)
    en.e3corr = -f.power * en.ehf3 / 2.0
    en.ehf1 = w * np.sum(f.b1 * (rt * t0) - f.b1p * (rn * tau[0] + rp * tau[1]))
    # energies.py:157-167 index the current with [:, :, :, c, s] (diagnostic only; restated as is)
    en.ehfCj0 = -w * np.sum(f.Ctau0 * ((cur[:, :, :, 0, 0] + cur[:, :, :, 0, 1]) ** 2
                                       + (cur[:, :, :, 1, 0] + cur[:, :, :, 1, 1]) ** 2
                                       + (cur[:, :, :, 2, 0] + cur[:, :, :, 2, 1]) ** 2))
    en.ehfCj1 = -w * np.sum(f.Ctau1 * ((-cur[:, :, :, 0, 0] + cur[:, :, :, 0, 1]) ** 2
                                       + (-cur[:, :, :, 1, 0] + cur[:, :, :, 1, 1]) ** 2
                                       + (-cur[:, :, :, 2, 0] + cur[:, :, :, 2, 1]) ** 2))
    divj = np.stack([sum(apply_along(D1[a], so[iq, a], a) for a in range(3)) for iq in range(2)])
    ehfls = w * np.sum(-f.b4 * rt * (divj[0] + divj[1]) - f.b4p * (rp * divj[1] + rn * divj[0]))
    en.ehfCdJ0 = w * np.sum(f.CdJ0 * rt * (divj[0] + divj[1]))
    en.ehfCdJ1 = w * np.sum(f.CdJ1 * r1 * (-divj[0] + divj[1]))
    cc = np.stack([np.stack([apply_along(D1[1], cur[iq, 2], 1) - apply_along(D1[2], cur[iq, 1], 2),
                             apply_along(D1[2], cur[iq, 0], 2) - apply_along(D1[0], cur[iq, 2], 0),
                             apply_along(D1[0], cur[iq, 1], 0) - apply_along(D1[1], cur[iq, 0], 1)])
                   for iq in range(2)])
    ctot = cc[0] + cc[1]
    en.ehflsodd = w * np.sum(-f.b4 * np.sum((sd[0] + sd[1]) * ctot, axis=0)
                             - f.b4p * np.sum(sd[0] * cc[0] + sd[1] * cc[1], axis=0))
    en.ehfls = ehfls + en.ehflsodd
    en.ehfc = 0.0
    en.ecorc = 0.0
    if tcoul:
        sc = -3.0 / 4.0 * f.slate if f.ex != 0 else 0.0
        en.ehfc = w * np.sum(0.5 * rp * coulomb.wcoul + sc * rp ** (4.0 / 3.0))
        en.ecorc = w * np.sum(sc / 3.0 * rp ** (4.0 / 3.0))
    en.ehft = w * np.sum(f.h2m[0] * tau[0] + f.h2m[1] * tau[1])
    en.e_zpe = 17.3 / levels.mass_number ** 0.2 if f.zpe == 1 else 0.0
    en.ehfint = (en.ehft + en.ehf0 + en.ehf1 + en.ehf2 + en.ehf3 + en.ehfls + en.ehfc
                 - np.sum(pairs.epair) - en.e_zpe)
    return en


def sum_energy(en, levels, mf, pairs):
    """E_bind from single-particle sums (energies.py:309-372)."""
    ww = levels.wocc * levels.wstates
    en.ehf = (np.sum(ww * (levels.sp_kinetic + levels.sp_energy)) / 2.0 + en.e3corr + mf.ecorrp
              + en.ecorc - np.sum(pairs.epair) - en.e_zpe)
    en.tke = np.sum(ww * levels.sp_kinetic)
    en.orbital = np.array([np.sum(ww * levels.sp_orbital[:, i]) for i in range(3)])
    en.spin = np.array([np.sum(ww * levels.sp_spin[:, i]) for i in range(3)])
    en.total_angmom = en.orbital + en.spin
    return en


def sp_properties(forces, grids, levels, cmtot=(0.0, 0.0, 0.0)):
    """Per-state kinetic energy, spin, orbital angular momentum, parity
    (inout.py:64-150)."""
    psi = levels.psi
    w = grids.wxyz
    xx = (grids.x - cmtot[0])[None, :, None, None]
    yy = (grids.y - cmtot[1])[None, None, :, None]
    zz = (grids.z - cmtot[2])[None, None, None, :]
    k2 = k2_total(grids)[None, None]
    h2m = np.where(levels.isospin == 0, forces.h2m[0], forces.h2m[1])
    kin = np.zeros(levels.nstmax)
    orb = np.zeros((levels.nstmax, 3))
    spin = np.zeros((levels.nstmax, 3))
    par = np.zeros(levels.nstmax)

    def part(sl):
        # states of ``sl``: writes disjoint entries
        ps = psi[sl]
        lap = np.fft.ifftn(np.fft.fftn(ps, axes=(2, 3, 4)) * k2, axes=(2, 3, 4))
        kin[sl] = w * h2m[sl] * -np.sum((np.conj(ps) * lap).real, axis=(1, 2, 3, 4))
        for i in range(sl.start, sl.stop):
            pst = psi[i]
            px, _ = cderv01(grids.dx, pst, 1)
            py, _ = cderv01(grids.dy, pst, 2)
            pz, _ = cderv01(grids.dz, pst, 3)
            re, im = pst.real, pst.imag
            orb[i] = w * np.array([
                np.sum(re * (yy[0] * pz.imag - zz[0] * py.imag) + im * (zz[0] * py.real - yy[0] * pz.real)),
                np.sum(re * (zz[0] * px.imag - xx[0] * pz.imag) + im * (xx[0] * pz.real - zz[0] * px.real)),
                np.sum(re * (xx[0] * py.imag - yy[0] * px.imag) + im * (yy[0] * px.real - xx[0] * py.real))])
            a, b = pst[0], pst[1]
            spin[i] = w * 0.5 * np.array([
                np.sum((np.conj(a) * b).real + (np.conj(b) * a).real),
                np.sum((np.conj(a) * b * (-1j)).real + (np.conj(b) * a * 1j).real),
                np.sum((np.conj(a) * a).real - (np.conj(b) * b).real)])
            fl = pst[:, ::-1, ::-1, ::-1]
            par[i] = w * np.sum(re * fl.real + im * fl.imag)

    pool.pmap(part, pool.chunks(0, levels.nstmax))
    levels.sp_kinetic = kin
    levels.sp_orbital, levels.sp_spin, levels.sp_parity = orb, spin, par
    return levels


def rms_radii(dens, grids):
    """Point rms radius per isospin about its own centre of mass
    (output.py:187-226, 246).  Returns ``(rms[2], rmstot)``."""
    w = grids.wxyz
    rms = np.zeros(2)
    pnr = np.zeros(2)
    coords = (grids.x[:, None, None], grids.y[None, :, None], grids.z[None, None, :])
    for iq in range(2):
        r = dens.rho[iq]
        pnr[iq] = np.sum(r) * w
        cm = [np.sum(c * r) * w / pnr[iq] for c in coords]
        r2 = sum((c - m) ** 2 for c, m in zip(coords, cm))
        rms[iq] = np.sqrt(np.sum(r2 * r) * w / pnr[iq])
    rmstot = np.sqrt((pnr[0] * rms[0] ** 2 + pnr[1] * rms[1] ** 2) / (pnr[0] + pnr[1]))
    return rms, rmstot


def observables(rho, grids, nneut, nprot, current=None):
    """Density part of calculate_complete_observables (output.py:177-276,
    323-340): particle numbers, centres of mass, summed currents, point rms
    radii and second moments about each isospin's own centre of mass, the
    quadrupole tensors Q_ij = sum (3 x_i x_j - delta_ij r^2) rho dV, Q20 /
    Q22 from their eigenvalues, the deformation beta / gamma and the
    isovector dipole.  Returns a dict keyed by the reference's field names."""
    w = grids.wxyz
    coords = (grids.x[:, None, None], grids.y[None, :, None], grids.z[None, None, :])
    pnr = np.zeros(2)
    cm = np.zeros((3, 2))
    pcm = np.zeros((3, 2))
    rms = np.zeros(2)
    x2m = np.zeros((3, 2))
    qmat = np.zeros((3, 3, 2))
    for iq in range(2):
        r = rho[iq]
        pnr[iq] = np.sum(r) * w
        for d in range(3):
            cm[d, iq] = np.sum(coords[d] * r) * w / pnr[iq]
            if current is not None:
                pcm[d, iq] = np.sum(current[iq, d]) * w
        rel = [coords[d] - cm[d, iq] for d in range(3)]
        r2 = rel[0] ** 2 + rel[1] ** 2 + rel[2] ** 2
        rms[iq] = np.sqrt(np.sum(r2 * r) * w / pnr[iq])
        for d in range(3):
            x2m[d, iq] = np.sum(rel[d] ** 2 * r) * w / pnr[iq]
        for i in range(3):
            for j in range(3):
                f = 3 * rel[i] ** 2 - r2 if i == j else 3 * rel[i] * rel[j]
                qmat[i, j, iq] = np.sum(f * r) * w
    pnrtot = pnr[0] + pnr[1]
    cmtot = (pnr[0] * cm[:, 0] + pnr[1] * cm[:, 1]) / pnrtot
    rmstot = np.sqrt((pnr[0] * rms[0] ** 2 + pnr[1] * rms[1] ** 2) / pnrtot)
    x2mtot = (pnr[0] * x2m[:, 0] + pnr[1] * x2m[:, 1]) / pnrtot
    c20, c22 = np.sqrt(5.0 / (16.0 * np.pi)), np.sqrt(5.0 / (96.0 * np.pi))
    q20, q22 = np.zeros(2), np.zeros(2)
    for iq in range(2):
        ev = np.linalg.eigvalsh(qmat[:, :, iq])
        q20[iq] = c20 * ev[2]
        q22[iq] = c22 * (ev[1] - ev[0])
    ev = np.linalg.eigvalsh(qmat[:, :, 0] + qmat[:, :, 1])
    q20tot, q22tot = c20 * ev[2], c22 * (ev[1] - ev[0])
    q20T1 = -q20[0] / nneut + q20[1] / nprot
    scale = 4.0 * np.pi / (5.0 * rmstot ** 2 * pnrtot)
    beta20tot, beta22tot = q20tot * scale, q22tot * scale
    beta = np.sqrt(beta20tot ** 2 + 2.0 * beta22tot ** 2)
    gamma = abs(np.arctan2(np.sqrt(2.0) * beta22tot, beta20tot)) * 180.0 / np.pi
    if gamma > 120.0:
        gamma -= 120.0
    if 60.0 < gamma <= 120.0:
        gamma = 120.0 - gamma
    dip = np.array([np.sum(coords[d] * (rho[0] / pnr[0] - rho[1] / pnr[1])) * w for d in range(3)])
    return dict(pnr=pnr, pnrtot=pnrtot, cm=cm, cmtot=cmtot, dipole_isovector=dip, rms=rms, rmstot=rmstot,
                x2m=x2m, x2mtot=x2mtot, q20=q20, q22=q22, q20tot=q20tot, q22tot=q22tot, q20T1=q20T1,
                beta20tot=beta20tot, beta22tot=beta22tot, beta=beta, gamma=gamma, pcm=pcm)
