"""Cartesian grid (mirror of grids.py:66-138) and the device context.

The dense derivative matrices der1/der2 (grids.py:36-61) and the Coulomb
Green's function live in the library context owned by the grid.
"""
from dataclasses import dataclass

import torch

from ._lib import Context


@dataclass
class Grids:
    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float
    periodic: bool
    wxyz: float
    x: torch.Tensor
    y: torch.Tensor
    z: torch.Tensor
    ctx: Context

    @property
    def n3(self):
        return self.nx * self.ny * self.nz


def init_grids(params=None, **kwargs):
    """grids.py:66-138 (Bloch phases / TABC are unimplemented stubs in the
    reference and raise here when requested)."""
    kw = dict(nx=48, ny=48, nz=48, dx=0.8, dy=0.8, dz=0.8, bangx=0.0, bangy=0.0, bangz=0.0, tabc_x=0,
              tabc_y=0, tabc_z=0, periodic=False)
    kw.update(kwargs)
    if any(abs(kw[b]) > 0.00001 for b in ("bangx", "bangy", "bangz")) and params is not None and not params.tfft:
        raise ValueError("bloch boundaries cannot be used without tfft.")
    if any(kw[t] != 0 for t in ("tabc_x", "tabc_y", "tabc_z")):
        raise ValueError("no tabc possible with tabc_nprocs=1.")
    if kw["nx"] % 2 or kw["ny"] % 2 or kw["nz"] % 2:
        raise ValueError("grids: nx, ny, and nz must be even.")
    if kw["dx"] * kw["dy"] * kw["dz"] <= 0.0:
        if kw["dx"] <= 0.0:
            raise ValueError("grid spacing given as 0.")
        kw["dy"] = kw["dz"] = kw["dx"]
    dev = torch.device("cuda")

    def centred(n, d):
        return (torch.arange(n, dtype=torch.float64, device=dev) - (n - 1) / 2.0) * d

    ctx = Context((kw["nx"], kw["ny"], kw["nz"]), (kw["dx"], kw["dy"], kw["dz"]), kw["periodic"],
                  kwargs.get("nstmax", 0))
    return Grids(nx=kw["nx"], ny=kw["ny"], nz=kw["nz"], dx=kw["dx"], dy=kw["dy"], dz=kw["dz"],
                 periodic=bool(kw["periodic"]), wxyz=kw["dx"] * kw["dy"] * kw["dz"],
                 x=centred(kw["nx"], kw["dx"]), y=centred(kw["ny"], kw["dy"]), z=centred(kw["nz"], kw["dz"]),
                 ctx=ctx)
