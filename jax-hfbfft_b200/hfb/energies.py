"""Energies (mirror of energies.py), evaluated on the device.

``Energies.dev`` holds the HFB_E_* values of the last integ_energy /
sum_energy call; ``sync()`` copies them (and the fluctuation measures left by
diagstep) to host attributes with the reference's names.
"""
import torch

from ._lib import call, ptr, stream_ptr, ENERGY_KEYS, HFB_NE


class Energies:
    def __init__(self):
        self.dev = torch.zeros(HFB_NE, dtype=torch.float64, device="cuda")
        self.efluct_dev = torch.zeros(4, dtype=torch.float64, device="cuda")   # efluct1q[2], efluct2q[2]
        self.efluct1prev = 0.0
        self.efluct2prev = 0.0
        self.ehfprev = 0.0
        for k in ENERGY_KEYS:
            setattr(self, k, 0.0)
        self.efluct1 = [0.0]
        self.efluct2 = [0.0]
        self.efluct1q = [0.0, 0.0]
        self.efluct2q = [0.0, 0.0]

    def sync(self):
        """One device->host copy of all scalars (synchronises the stream)."""
        both = torch.cat([self.dev, self.efluct_dev]).cpu().tolist()
        for k, v in zip(ENERGY_KEYS, both[:HFB_NE]):
            setattr(self, k, v)
        q = both[HFB_NE:]
        self.efluct1q = q[0:2]
        self.efluct2q = q[2:4]
        # static.py:574-575
        self.efluct1 = [max(q[0], q[1])]
        self.efluct2 = [0.5 * (q[2] + q[3])]
        return self


def init_energies(**kwargs):
    e = Energies()
    for k, v in kwargs.items():
        setattr(e, k, v)
    return e


def integ_energy(coulomb, densities, energies, forces, grids, levels, params, pairs):
    """EDF integrals (energies.py:90-306) on the device; values land on
    ``energies.dev``."""
    d = densities
    call("hfb_energies", grids.ctx.handle, forces.c_struct(), int(bool(getattr(params, "tcoul", True))),
         float(levels.mass_number), ptr(d.rho), ptr(d.tau), ptr(d.current), ptr(d.sdens), ptr(d.sodens),
         ptr(coulomb.wcoul), ptr(pairs.out[1]), ptr(energies.dev), stream_ptr())
    return energies


def sum_energy(energies, levels, meanfield, pairs, grids=None):
    """E_bind from the single-particle sums (energies.py:309-372)."""
    lv = levels
    ctx = grids.ctx if grids is not None else _ctx_of(lv)
    call("hfb_sum_energy", ctx.handle, lv.nstmax, ptr(lv.wocc), ptr(lv.wstates), ptr(lv.sp_kinetic),
         ptr(lv.sp_energy), ptr(pairs.out[1]), ptr(meanfield.ecorrp_dev), ptr(energies.dev), stream_ptr())
    return energies


def _ctx_of(levels):
    ctx = getattr(levels, "_ctx", None)
    if ctx is None:
        raise RuntimeError("sum_energy needs the grid context: pass grids= or create levels with init_levels")
    return ctx
