"""Mean fields and the single-particle Hamiltonian (mirror of meanfield.py).

Besides the reference's arrays the mean field keeps ``pot``: the twelve
fields hpsi reads, packed [2][12][n^3] in the precision of the states.
"""
from dataclasses import dataclass

import torch

from ._lib import call, ptr, stream_ptr, prec_of, HFB_F64, HFB_F32


@dataclass
class Meanfield:
    upot: torch.Tensor
    bmass: torch.Tensor
    divaq: torch.Tensor
    v_pair: torch.Tensor
    aq: torch.Tensor
    spot: torch.Tensor
    wlspot: torch.Tensor
    dbmass: torch.Tensor
    ecorrp_dev: torch.Tensor
    pot: torch.Tensor

    @property
    def ecorrp(self):
        return float(self.ecorrp_dev[0])

    def pack(self, dtype):
        """Repack the hpsi potentials for states of ``dtype``."""
        rd = torch.float64 if dtype == torch.complex128 else torch.float32
        pot = torch.empty((2, 12) + tuple(self.upot.shape[1:]), dtype=rd, device=self.upot.device)
        pot[:, 0] = self.upot
        pot[:, 1] = self.bmass
        pot[:, 2] = self.v_pair
        pot[:, 3:6] = self.aq
        pot[:, 6:9] = self.spot
        pot[:, 9:12] = self.wlspot
        self.pot = pot
        return self


def init_meanfield(grids, dtype=torch.complex128):
    """meanfield.py:23-38."""
    dev = torch.device("cuda")
    s4 = (2, grids.nx, grids.ny, grids.nz)
    s5 = (2, 3, grids.nx, grids.ny, grids.nz)
    rd = torch.float64 if dtype == torch.complex128 else torch.float32
    z4 = lambda: torch.zeros(s4, dtype=torch.float64, device=dev)
    z5 = lambda: torch.zeros(s5, dtype=torch.float64, device=dev)
    return Meanfield(upot=z4(), bmass=z4(), divaq=z4(), v_pair=z4(), aq=z5(), spot=z5(), wlspot=z5(), dbmass=z5(),
                     ecorrp_dev=torch.zeros(1, dtype=torch.float64, device=dev),
                     pot=torch.zeros((2, 12) + s4[1:], dtype=rd, device=dev))


def hpsi01(grids, meanfield, iq, weight, weightuv, pinn):
    """h_q on a 2-spinor or a batch of spinors of one isospin
    (meanfield.py:41-159).  Returns ``(pout, pout_mf, pout_del)``."""
    x = pinn.contiguous()
    nst = x.numel() // (2 * grids.n3)
    rd = torch.float64 if x.dtype == torch.complex128 else torch.float32
    if meanfield.pot.dtype != rd:
        meanfield.pack(x.dtype)
    dev = x.device
    wt = torch.as_tensor(weight, dtype=torch.float64, device=dev).reshape(-1).expand(nst).contiguous()
    wu = torch.as_tensor(weightuv, dtype=torch.float64, device=dev).reshape(-1).expand(nst).contiguous()
    pout = torch.empty_like(x)
    pmf = torch.empty_like(x)
    pdel = torch.empty_like(x)
    nneut = 0 if iq == 1 else nst
    call("hfb_hpsi", grids.ctx.handle, prec_of(x), ptr(meanfield.pot), nst, nneut, ptr(x), ptr(wt), ptr(wu),
         ptr(pout), ptr(pmf), ptr(pdel), stream_ptr())
    return pout, pmf, pdel


def skyrme(coulomb, densities, forces, grids, meanfield, params, static, constraints=None, dtype=None):
    """Potentials from densities (meanfield.py:164-391), on the device.
    With ``constraints`` (hfb.constraint.Constraints) the constraint
    potential is subtracted from upot afterwards, where meanfield.py:246-248
    leaves the place for it."""
    if getattr(static, "outertype", "N") != "N":
        raise NotImplementedError(f"outertype '{static.outertype}' not implemented.")
    if dtype is None:
        dtype = torch.complex128 if meanfield.pot.dtype == torch.float64 else torch.complex64
    rd = torch.float64 if dtype == torch.complex128 else torch.float32
    if meanfield.pot.dtype != rd:
        meanfield.pot = torch.empty(meanfield.pot.shape, dtype=rd, device=meanfield.pot.device)
    fs = forces.c_struct()
    d, m = densities, meanfield
    tcoul = bool(getattr(params, "tcoul", True))
    call("hfb_skyrme", grids.ctx.handle, fs, int(tcoul), ptr(d.rho), ptr(d.tau), ptr(d.chi), ptr(d.current),
         ptr(d.sdens), ptr(d.sodens), ptr(m.upot), ptr(m.bmass), ptr(m.divaq), ptr(m.v_pair), ptr(m.aq),
         ptr(m.spot), ptr(m.wlspot), ptr(m.dbmass), ptr(coulomb.wcoul), ptr(m.ecorrp_dev),
         HFB_F64 if rd == torch.float64 else HFB_F32, ptr(m.pot), stream_ptr())
    if constraints is not None:
        from .constraint import add_constraint_potential
        add_constraint_potential(meanfield, constraints, grids)
    return meanfield, coulomb
