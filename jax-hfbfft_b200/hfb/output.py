"""Radii, the nuclear observables (output.py:177-340) and the reference's
.res output files (output.py:49-174)."""
import os
from dataclasses import dataclass

import numpy as np
import torch

from ._lib import call, ptr, stream_ptr


def rms_radii(densities, grids):
    """Point rms radius per isospin about its own centre of mass and the
    total (output.py:187-226, 246).  Returns (pnr[2], rms[2], rmstot)."""
    out = torch.zeros(5, dtype=torch.float64, device="cuda")
    call("hfb_rms", grids.ctx.handle, ptr(densities.rho), ptr(out), stream_ptr())
    v = out.cpu().tolist()
    return v[0:2], v[2:4], v[4]


# Layout of hfb_observables' output (include/hfb.h, HFB_OBS_*): name ->
# (offset, shape).
_OBS = dict(pnr=(0, (2,)), cm=(2, (3, 2)), pcm=(8, (3, 2)), rms=(14, (2,)), x2m=(16, (3, 2)), q20=(22, (2,)),
            q22=(24, (2,)), pnrtot=(26, ()), cmtot=(27, (3,)), rmstot=(30, ()), x2mtot=(31, (3,)), q20tot=(34, ()),
            q22tot=(35, ()), q20T1=(36, ()), beta20tot=(37, ()), beta22tot=(38, ()), beta=(39, ()), gamma=(40, ()),
            dipole_isovector=(41, (3,)), qmat=(44, (3, 3, 2)))
HFB_NOBS = 62


@dataclass
class CompleteNuclearObservables:
    """The reference's CompleteNuclearObservables (output.py:8-46) plus
    ``qmat``, the per-isospin quadrupole tensors (3, 3, 2).  The angular
    momenta are the occupation-weighted sums of the levels' single-particle
    orbital and spin expectation values (output.py:297-320); they are zero
    while nothing has filled ``levels.sp_orbital`` / ``sp_spin``."""
    pnr: np.ndarray
    pnrtot: float
    cm: np.ndarray
    cmtot: np.ndarray
    dipole_isovector: np.ndarray
    rms: np.ndarray
    rmstot: float
    x2m: np.ndarray
    x2mtot: np.ndarray
    q20: np.ndarray
    q22: np.ndarray
    q20tot: float
    q22tot: float
    q20T1: float
    beta20tot: float
    beta22tot: float
    beta: float
    gamma: float
    pcm: np.ndarray
    qmat: np.ndarray
    orbital_momentum: np.ndarray = None
    spin_momentum: np.ndarray = None
    total_momentum: np.ndarray = None


def observables_raw(grids, rho, nneut, nprot, current=None):
    """hfb_observables on device densities: the HFB_NOBS raw values as a
    CUDA FP64 tensor (no host synchronisation)."""
    if rho.dtype != torch.float64 or (current is not None and current.dtype != torch.float64):
        raise TypeError("observables need FP64 densities")
    out = torch.empty(HFB_NOBS, dtype=torch.float64, device=rho.device)
    call("hfb_observables", grids.ctx.handle, ptr(rho.contiguous()),
         None if current is None else ptr(current.contiguous()), float(nneut), float(nprot), ptr(out), stream_ptr())
    return out


def calculate_complete_observables(densities, levels, grids, params=None, current_densities=None):
    """output.py:177-340 (density part): particle numbers, centres of mass,
    radii, second moments, quadrupole moments and deformation, isovector
    dipole and, with ``current_densities`` ([2, 3, n, n, n]), the summed
    currents ``pcm``.  One device reduction, one copy to the host."""
    v = observables_raw(grids, densities.rho, levels.nneut, levels.nprot, current_densities).cpu().numpy()
    vals = {}
    for k, (o, shp) in _OBS.items():
        n = int(np.prod(shp)) if shp else 1
        x = v[o:o + n]
        vals[k] = float(x[0]) if not shp else x.reshape(shp).copy()
    vals["orbital_momentum"], vals["spin_momentum"] = angular_momentum(levels)
    vals["total_momentum"] = vals["orbital_momentum"] + vals["spin_momentum"]
    return CompleteNuclearObservables(**vals)


def angular_momentum(levels):
    """Occupation-weighted sums of the single-particle orbital and spin
    expectation values over states with wocc > 1e-10 (output.py:297-320);
    zeros for levels without them."""
    orb, spin = getattr(levels, "sp_orbital", None), getattr(levels, "sp_spin", None)
    if orb is None or spin is None:
        return np.zeros(3), np.zeros(3)
    w = levels.wocc * levels.wstates * (levels.wocc > 1e-10)
    orb = orb if orb.shape[-1] == 3 else orb.T   # (nst, 3)
    spin = spin if spin.shape[-1] == 3 else spin.T
    return (w[:, None] * orb).sum(0).cpu().numpy(), (w[:, None] * spin).sum(0).cpu().numpy()


class FortranOutputWriter:
    """The reference's per-iteration .res files (output.py:49-174): the same
    file names, header lines and column formats, so that tools reading the
    reference's (and the Fortran code's) output read these.  Files are
    created with their headers when the writer is made and get one line per
    ``write_iteration_data`` call."""

    HEADERS = {
        "conver": "# Iter   Energy  d_Energy    sp_fluct    max(lam-)     rms(lam-)      rms    "
                  "beta2  gamma      x_0     e_pair(1)    e_pair(2)\n",
        "energies": "# Iter    N(n)    N(p)       E(sum)         E(integ)       Ekin         "
                    "E_Coul         ehfCrho0       ehfCrho1       ehfCdrho0      ehfCdrho1     "
                    "ehfCtau0       ehfCtau1       ehfCdJ0        ehfCdJ1       e_pair(1)    "
                    "e_pair(2)      e_zpe\n",
        "dipoles": "# Iter    c.m. x-y-z                                  Isovector dipoles x-y-z\n",
        "spin": "# Iter      Lx        Ly        Lz        Sx        Sy        Sz        Jx        Jy        Jz\n",
        "monopoles": "# Iter    RMS_n     RMS_p     RMS_tot   RMS_diff   N_dens    Z_dens    A_dens\n",
        "quadrupoles": "# Iter    Q20_n     Q20_p     Q20_tot   Q22_tot   <x\u00b2>_tot  <y\u00b2>_tot  "
                       "<z\u00b2>_tot  Beta      Gamma\n",
        "momenta": "# Iter    Px_n      Py_n      Pz_n      Px_p      Py_p      Pz_p      "
                   "Px_tot    Py_tot    Pz_tot\n",
    }

    def __init__(self, output_dir):
        self.output_dir = output_dir
        os.makedirs(output_dir, exist_ok=True)
        self.files = {k: os.path.join(output_dir, f"{k}.res") for k in self.HEADERS}
        for k, h in self.HEADERS.items():
            with open(self.files[k], "w", encoding="utf-8") as f:
                f.write(h)

    def _append(self, key, text):
        with open(self.files[key], "a", encoding="utf-8") as f:
            f.write(text + "\n")

    def write_iteration_data(self, iteration, energies, observables, static, pairs):
        en, ob, ep = energies, observables, pairs.epair
        de = 0.0
        if getattr(en, "ehfprev", 0.0) != 0.0 and iteration > 0:
            de = en.ehf - en.ehfprev
        f1, f2 = en.efluct1[0], en.efluct2[0]
        self._append("conver", f"{iteration:4d} {en.ehf:12.6f} {de:12.6f} {f1:12.6e} {f1:12.6e} {f2:12.6e} "
                               f"{ob.rmstot:8.4f} {ob.beta:8.4f} {ob.gamma:8.2f} {static.x0dmp:8.4f} "
                               f"{ep[0]:12.6f} {ep[1]:12.6f}")
        cols = [en.ehfCrho0, en.ehfCrho1, en.ehfCdrho0, en.ehfCdrho1, en.ehfCtau0, en.ehfCtau1, en.ehfCdJ0,
                en.ehfCdJ1, ep[0], ep[1], en.e_zpe]
        self._append("energies", f"{iteration:4d} {ob.pnr[0]:8.2f} {ob.pnr[1]:8.2f} {en.ehf:14.6f} "
                                 f"{en.ehfint:14.6f} {en.tke:12.6f} {en.ehfc:12.6f} "
                                 + " ".join(f"{c:12.6f}" for c in cols))
        self._append("dipoles", f"{iteration:4d} " + " ".join(f"{c:12.6f}" for c in list(ob.cmtot[:3])
                                                             + list(ob.dipole_isovector[:3])))
        mom = list(ob.orbital_momentum[:3]) + list(ob.spin_momentum[:3]) + list(ob.total_momentum[:3])
        self._append("spin", f"{iteration:4d} " + " ".join(f"{c:10.6f}" for c in mom))
        self._append("monopoles", f"{iteration:4d} {ob.rms[0]:9.6f} {ob.rms[1]:9.6f} {ob.rmstot:9.6f} "
                                  f"{ob.rms[0] - ob.rms[1]:9.6f} {ob.pnr[0]:9.3f} {ob.pnr[1]:9.3f} "
                                  f"{ob.pnrtot:9.3f}")
        self._append("quadrupoles", f"{iteration:4d} " + " ".join(
            f"{c:9.6f}" for c in [ob.q20[0], ob.q20[1], ob.q20tot, ob.q22tot, ob.x2mtot[0], ob.x2mtot[1],
                                  ob.x2mtot[2], ob.beta]) + f" {ob.gamma:9.2f}")
        p = np.asarray(ob.pcm)
        self._append("momenta", f"{iteration:4d} " + " ".join(
            f"{c:10.6f}" for c in [p[0, 0], p[1, 0], p[2, 0], p[0, 1], p[1, 1], p[2, 1], p[0, 0] + p[0, 1],
                                  p[1, 0] + p[1, 1], p[2, 0] + p[2, 1]]))


def res_callback(state, writer, current=False):
    """A ``callback(i, energies)`` for hfb.static.statichf that appends one
    line per iteration to the .res files of ``writer``, as the reference's
    statichf_with_benchmark does with an output writer (static.py:1721-1733,
    complete_sinfo_with_fortran_output)."""
    def cb(i, energies):
        obs = calculate_complete_observables(state["densities"], state["levels"], state["grids"], state["params"],
                                             state["densities"].current if current else None)
        writer.write_iteration_data(i, energies, obs, state["static"], state["pairs"])
    return cb
