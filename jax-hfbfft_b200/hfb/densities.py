"""Local densities (mirror of densities.py)."""
from dataclasses import dataclass
import ctypes as C

import torch

from ._lib import call, ptr, stream_ptr, prec_of


@dataclass
class Densities:
    rho: torch.Tensor
    chi: torch.Tensor
    tau: torch.Tensor
    current: torch.Tensor
    sdens: torch.Tensor
    sodens: torch.Tensor


def init_densities(grids):
    dev = torch.device("cuda")
    s4 = (2, grids.nx, grids.ny, grids.nz)
    s5 = (2, 3, grids.nx, grids.ny, grids.nz)
    z = lambda s: torch.zeros(s, dtype=torch.float64, device=dev)
    return Densities(rho=z(s4), chi=z(s4), tau=z(s4), current=z(s5), sdens=z(s5), sodens=z(s5))


def add_density(densities, grids, levels, mix=1.0, forces=None):
    """densities.py:177-234.  ``mix`` < 1 blends rho, tau, chi with the
    previous values (static.py:1820-1823).  With ``forces`` given the
    per-state kinetic energies of inout.py:129-132 are refreshed from the
    same derivatives."""
    d, lv = densities, levels
    kin = None
    h2m = None
    if forces is not None:
        kin = lv.sp_kinetic
        h2m = (C.c_double * 2)(float(forces.h2m[0]), float(forces.h2m[1]))
    call("hfb_add_density", grids.ctx.handle, prec_of(lv.psi), lv.nstmax, lv.npsi[0], ptr(lv.psi), ptr(lv.wocc),
         ptr(lv.wguv), ptr(lv.pairwg), ptr(lv.wstates), float(mix), ptr(d.rho), ptr(d.chi), ptr(d.tau),
         ptr(d.current), ptr(d.sdens), ptr(d.sodens), h2m, ptr(kin), stream_ptr())
    return densities
