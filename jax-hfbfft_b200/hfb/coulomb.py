"""Coulomb potential (mirror of coulomb.py).  The Green's function on the
doubled grid is built on the device when the grid context is created."""
from dataclasses import dataclass

import torch

from ._lib import call, ptr, stream_ptr


@dataclass
class Coulomb:
    nx2: int
    ny2: int
    nz2: int
    wcoul: torch.Tensor


def init_coulomb(grids):
    """coulomb.py:23-52."""
    f = 1 if grids.periodic else 2
    return Coulomb(nx2=f * grids.nx, ny2=f * grids.ny, nz2=f * grids.nz,
                   wcoul=torch.zeros((grids.nx, grids.ny, grids.nz), dtype=torch.float64, device="cuda"))


def poisson(grids, params, coulomb, rho):
    """coulomb.py:54-75: potential of the proton density rho[1]."""
    rp = rho[1].contiguous().to(torch.float64)
    w = torch.empty((grids.nx, grids.ny, grids.nz), dtype=torch.float64, device=rp.device)
    call("hfb_poisson", grids.ctx.handle, ptr(rp), ptr(w), stream_ptr())
    return w
