"""Single-particle properties (mirror of inout.py:64-150), on the device:
the kinetic energy from the spectral derivatives (with the Nyquist term of
the full k^2 Laplacian), and the orbital angular momentum about the centre
of mass in ``moment.cmtot`` (the origin without one), the spin and the
parity of every state.
"""
import ctypes as C

from ._lib import call, ptr, stream_ptr, prec_of


def sp_properties(forces, grids, levels, moment=None):
    h2m = (C.c_double * 2)(float(forces.h2m[0]), float(forces.h2m[1]))
    call("hfb_sp_kinetic", grids.ctx.handle, prec_of(levels.psi), levels.nstmax, levels.npsi[0], ptr(levels.psi),
         h2m, ptr(levels.sp_kinetic), stream_ptr())
    cmt = getattr(moment, "cmtot", None) if moment is not None else None
    cm = None if cmt is None else (C.c_double * 3)(*[float(v) for v in cmt])
    call("hfb_sp_properties", grids.ctx.handle, prec_of(levels.psi), levels.nstmax, ptr(levels.psi), cm,
         ptr(levels.sp_orbital), ptr(levels.sp_spin), ptr(levels.sp_parity), stream_ptr())
    return levels
