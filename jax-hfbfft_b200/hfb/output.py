"""Radii and the density part of the nuclear observables (output.py:177-340)."""
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
    """The reference's CompleteNuclearObservables (output.py) without the
    angular-momentum fields, which need single-particle orbital and spin
    expectation values this library does not compute; ``qmat`` (the
    per-isospin quadrupole tensors, (3, 3, 2)) is added."""
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
    return CompleteNuclearObservables(**vals)
