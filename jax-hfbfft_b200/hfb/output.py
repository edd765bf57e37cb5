"""Radii (the subset of output.py:177-246 the metric needs)."""
import torch

from ._lib import call, ptr, stream_ptr


def rms_radii(densities, grids):
    """Point rms radius per isospin about its own centre of mass and the
    total (output.py:187-226, 246).  Returns (pnr[2], rms[2], rmstot)."""
    out = torch.zeros(5, dtype=torch.float64, device="cuda")
    call("hfb_rms", grids.ctx.handle, ptr(densities.rho), ptr(out), stream_ptr())
    v = out.cpu().tolist()
    return v[0:2], v[2:4], v[4]
