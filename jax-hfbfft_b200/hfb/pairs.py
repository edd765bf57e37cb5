"""BCS pairing (mirror of pairs.py), solved on the device."""
from dataclasses import dataclass, field
import math

import torch

from ._lib import call, ptr, stream_ptr, PairArgs


@dataclass
class Pairs:
    out: torch.Tensor = field(default_factory=lambda: torch.zeros((5, 2), dtype=torch.float64, device="cuda"))
    firstcall: bool = True

    # eferm, epair, avdelt, avdeltv2, avg (pairs.py:15-22)
    @property
    def eferm(self):
        return self.out[0]

    @property
    def epair(self):
        return self.out[1]

    @property
    def avdelt(self):
        return self.out[2]

    @property
    def avdeltv2(self):
        return self.out[3]

    @property
    def avg(self):
        return self.out[4]


def pair(levels, meanfield, forces, params, grids, pairs):
    """pairs.py:161-220: gap (constant 11.2/sqrt(A) while iteration <= 10,
    else the diagonal of the gap matrix left by diagstep), Fermi level by
    Brent's method, soft cutoffs, v^2 and uv.  Device errors (no bracket)
    surface at the next status check."""
    if params.iteration > 10 and pairs.firstcall:
        raise NotImplementedError("pairing gap from <v_pair> (pairs.py:143-157) is only reached on a restart")
    lv = levels
    a = PairArgs()
    a.npsi[0], a.npsi[1] = lv.npsi
    a.nneut, a.nprot = lv.nneut, lv.nprot
    a.use_const_gap = int(params.iteration <= 10)
    a.const_gap = 11.2 / math.sqrt(lv.mass_number)
    a.pair_cutoff[0], a.pair_cutoff[1] = forces.pair_cutoff
    a.state_cutoff[0], a.state_cutoff[1] = forces.state_cutoff
    a.softcut_range = float(forces.softcut_range)
    a.sp_energy = ptr(lv.sp_energy)
    a.deltaf, a.wocc, a.wguv, a.pairwg, a.wstates = (ptr(lv.deltaf), ptr(lv.wocc), ptr(lv.wguv), ptr(lv.pairwg),
                                                     ptr(lv.wstates))
    a.out = ptr(pairs.out)
    call("hfb_pair", grids.ctx.handle, a, stream_ptr())
    pairs.firstcall = False
    return levels, pairs
