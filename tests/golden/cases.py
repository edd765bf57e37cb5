"""Small end-to-end cases shared by the golden generator and the tests.

Each case is run by the reference driver (``statichf_with_benchmark``) in
``make_golden.py`` and by the oracle / CUDA path in the tests.  ``static``
follows the reference's _config.yml defaults (inibcs = inidiag = 30) unless
set here.
"""

RUN_CASES = {
    # O16-like, no pairing: 40 iterations cross the inibcs switch (tbcs -> False).
    "o16_n16": dict(grid=dict(nx=16, ny=16, nz=16, dx=1.0, dy=1.0, dz=1.0),
                    force=dict(name="SLy4", ipair=0, tbcs=False),
                    levels=dict(nneut=8, nprot=8, npsi=[10, 10]),
                    static=dict(maxiter=40, radinx=2.26, radiny=2.26, radinz=2.26, serr=1e-20,
                                x0dmp=0.2, e0dmp=100.0, tvaryx_0=True, iternat=0),
                    mprint=1),
    # Ne20-like, volume-delta pairing with a 60 MeV soft pairing window, deformed start.
    "ne20_vdi_n16": dict(grid=dict(nx=16, ny=16, nz=16, dx=1.0, dy=1.0, dz=1.0),
                         force=dict(name="SLy4", ipair=5, tbcs=True, v0prot=300.0, v0neut=300.0,
                                    pair_cutoff=[60.0, 60.0]),
                         levels=dict(nneut=10, nprot=10, npsi=[14, 14]),
                         static=dict(maxiter=16, radinx=2.3, radiny=2.3, radinz=2.7, serr=1e-20,
                                     x0dmp=0.2, e0dmp=100.0, tvaryx_0=True, iternat=0),
                         mprint=1),
    # DDDI pairing with a state cutoff, as in the reference's _config.yml (smaller box).
    "o18_dddi_n16": dict(grid=dict(nx=16, ny=16, nz=16, dx=1.0, dy=1.0, dz=1.0),
                         force=dict(name="SLy4", ipair=6, tbcs=True, v0prot=362.0, v0neut=362.0,
                                    rho0pr=0.32, state_cutoff=[15.0, 15.0]),
                         levels=dict(nneut=10, nprot=8, npsi=[14, 12]),
                         static=dict(maxiter=14, radinx=2.3, radiny=2.3, radinz=2.3, serr=1e-20,
                                     x0dmp=0.45, e0dmp=100.0, tvaryx_0=True, iternat=0),
                         mprint=1),
}


# The bench workloads (hfb.config presets, same inputs on both sides) run by
# the reference driver for a bounded number of iterations: O16 (24^3, 10 + 10
# states, no pairing) to the workload's iteration cap of 500, Cr48 (32^3,
# 32 + 32 states, VDI, beta = 0.2) for its first 20 iterations, Pb208 (48^3,
# 140 + 96 states, VDI) for its first 3.  The fixtures keep per-iteration
# scalars, final single-particle quantities, radii and the inputs and
# outputs of the reference's post-loop lastdiag -- no states, so they stay
# small.
CONFIG_RUNS = {
    "o16_n24": dict(workload="O16", maxiter=500),
    "cr48_n32": dict(workload="Cr48", maxiter=20),
    "pb208_n48": dict(workload="Pb208", maxiter=3),
}
