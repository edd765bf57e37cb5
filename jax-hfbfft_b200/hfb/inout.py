"""Single-particle properties (mirror of inout.py:64-150).

The energy functional needs only ``sp_kinetic``; it is computed on the
device from the spectral derivatives (with the Nyquist term of the full k^2
Laplacian).  Orbital angular momentum, spin and parity are printout-only in
the reference and are not computed here.
"""
import ctypes as C

from ._lib import call, ptr, stream_ptr, prec_of


def sp_properties(forces, grids, levels, moment=None):
    h2m = (C.c_double * 2)(float(forces.h2m[0]), float(forces.h2m[1]))
    call("hfb_sp_kinetic", grids.ctx.handle, prec_of(levels.psi), levels.nstmax, levels.npsi[0], ptr(levels.psi),
         h2m, ptr(levels.sp_kinetic), stream_ptr())
    return levels
