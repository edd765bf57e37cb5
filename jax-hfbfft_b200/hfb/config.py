"""Workload presets and the set-up sequence of the reference's run_hfb
(test.py:121-166).

Oscillator seeds: hbar*omega = 41 A^(-1/3) MeV, b^2 = 2 h2m / (hbar omega)
with the unscaled h2m of the force, and the reference's Gaussian
exp(-x^2 / radin^2) so radin = sqrt(2) b.  A quadrupole deformation beta
stretches z and squeezes x, y at fixed volume:
radin_z = radin exp(c beta), radin_x = radin_y = radin exp(-c beta / 2),
c = sqrt(5 / (4 pi)).
Pairing strengths follow the reference's sign convention (positive v0,
the attraction carried by -weightuv * v_pair, meanfield.py:155-157).
"""
import copy
import math

import torch

WORKLOADS = {
    # 24^3, dx 1.0, 10 + 10 states, N = Z = 8, no pairing
    "O16": dict(grid=dict(nx=24, ny=24, nz=24, dx=1.0, dy=1.0, dz=1.0),
                force=dict(name="SLy4", ipair=0, tbcs=False),
                levels=dict(nneut=8, nprot=8, npsi=[10, 10]),
                static=dict(maxiter=500, serr=1e-20, x0dmp=0.2, e0dmp=100.0, tvaryx_0=True),
                beta=0.0, mprint=1),
    # 32^3, dx 0.8, 32 + 32 states, N = Z = 24, volume delta pairing, 60 MeV window, beta = 0.2
    "Cr48": dict(grid=dict(nx=32, ny=32, nz=32, dx=0.8, dy=0.8, dz=0.8),
                 force=dict(name="SLy4", ipair=5, tbcs=True, v0prot=300.0, v0neut=300.0, pair_cutoff=[60.0, 60.0]),
                 levels=dict(nneut=24, nprot=24, npsi=[32, 32]),
                 static=dict(maxiter=1000, serr=1e-20, x0dmp=0.2, e0dmp=100.0, tvaryx_0=True),
                 beta=0.2, mprint=1),
    # 48^3, dx 0.8, 140 + 96 states, N = 126, Z = 82, volume delta pairing (force table strengths)
    "Pb208": dict(grid=dict(nx=48, ny=48, nz=48, dx=0.8, dy=0.8, dz=0.8),
                  force=dict(name="SLy4", ipair=5, tbcs=True, pair_cutoff=[60.0, 60.0]),
                  levels=dict(nneut=126, nprot=82, npsi=[140, 96]),
                  static=dict(maxiter=2000, serr=1e-20, x0dmp=0.2, e0dmp=100.0, tvaryx_0=True),
                  beta=0.0, mprint=1),
    # 32^3, dx 0.8, 40 + 30 states, N = 28, Z = 20, volume delta pairing
    "Ca48": dict(grid=dict(nx=32, ny=32, nz=32, dx=0.8, dy=0.8, dz=0.8),
                 force=dict(name="SLy4", ipair=5, tbcs=True, pair_cutoff=[60.0, 60.0]),
                 levels=dict(nneut=28, nprot=20, npsi=[40, 30]),
                 static=dict(maxiter=1000, serr=1e-20, x0dmp=0.2, e0dmp=100.0, tvaryx_0=True),
                 beta=0.0, mprint=1),
}


def ho_radii(nneut, nprot, h2m=20.735530, beta=0.0):
    a = nneut + nprot
    hw = 41.0 * a ** (-1.0 / 3.0)
    radin = math.sqrt(2.0) * math.sqrt(2.0 * h2m / hw)
    c = math.sqrt(5.0 / (4.0 * math.pi))
    return radin * math.exp(-0.5 * c * beta), radin * math.exp(-0.5 * c * beta), radin * math.exp(c * beta)


def case_dict(name, **over):
    """A deep copy of a preset with the oscillator radii filled in."""
    c = copy.deepcopy(WORKLOADS[name])
    for k, v in over.items():
        if isinstance(v, dict):
            c[k].update(v)
        else:
            c[k] = v
    st = c["static"]
    if "radinx" not in st:
        rx, ry, rz = ho_radii(c["levels"]["nneut"], c["levels"]["nprot"], beta=c.get("beta", 0.0))
        st.update(radinx=rx, radiny=ry, radinz=rz)
    return c


def setup(case, dtype=torch.complex128):
    """Build every state object for a case dict (the order of run_hfb,
    test.py:145-166) and seed the oscillator states."""
    from .params import init_params
    from .forces import init_forces
    from .grids import init_grids
    from .densities import init_densities
    from .meanfield import init_meanfield
    from .levels import init_levels
    from .static import init_static, harmosc
    from .coulomb import init_coulomb
    from .energies import init_energies
    from .pairs import Pairs
    params = init_params(imode=1, mprint=case.get("mprint", 1))
    forces = init_forces(params, **case["force"])
    grids = init_grids(params, **case["grid"])
    densities = init_densities(grids)
    meanfield = init_meanfield(grids, dtype)
    lv = case["levels"]
    levels = init_levels(grids, lv["nneut"], lv["nprot"], lv.get("npsi"), dtype=dtype)
    forces, static = init_static(forces, levels, **case["static"])
    coulomb = init_coulomb(grids)
    energies = init_energies()
    pairs = Pairs()
    levels = harmosc(grids, levels, params, static)
    return dict(coulomb=coulomb, densities=densities, energies=energies, forces=forces, grids=grids,
                levels=levels, meanfield=meanfield, moment=None, params=params, static=static, pairs=pairs)
