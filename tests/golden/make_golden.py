"""Generate golden vectors by running the jax-hfbfft reference modules themselves.

JAX is not installed in the build container, so the reference modules are
imported unmodified with ``tests/golden/jaxshim`` first on ``sys.path``: a
NumPy-backed stand-in for the subset of the jax API they use (see the
docstring of ``jaxshim/jax/__init__.py`` for the semantics restated).

Run from the repository root, in the build container only (it reads the
reference checkout)::

    python tests/golden/make_golden.py --ref <path of the reference checkout>

Outputs (committed): ``tests/golden/unit_n8.npz`` (per-function vectors on an
8^3 grid with seeded random inputs), ``tests/golden/run_<case>.npz``
(end-to-end runs of the reference driver ``statichf_with_benchmark`` on small
grids: per-iteration energies and final densities / levels) and
``tests/golden/observables_n16.npz`` (``calculate_complete_observables`` on
the runs' final densities and on a seeded triaxial density; needs the run
fixtures, ``--only observables`` regenerates it alone) and
``tests/golden/res_files.json`` (the text of the reference's .res writers
for seeded inputs, ``--only res``) and ``tests/golden/constraint_n16.npz``
(the reference's constraint module on seeded inputs, ``--only constraint``)
and ``tests/golden/config_<case>.npz`` (the bench workloads through the
reference driver for a bounded number of iterations, with its post-loop
``lastdiag``; ``--only config`` or ``--only <case>``) and
``tests/golden/natural_n8.npz`` (the reference's hfb_natural on seeded
inputs, ``--only natural``).
"""
import argparse
import contextlib
import io
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from cases import RUN_CASES, CONFIG_RUNS  # noqa: E402  (shared with the tests)


def _import_reference(ref):
    sys.path.insert(0, os.path.join(HERE, "jaxshim"))
    sys.path.insert(1, ref)
    import jax  # noqa: F401  (the stand-in)
    mods = {}
    for name in ("params", "forces", "grids", "densities", "meanfield", "levels", "static",
                 "coulomb", "moment", "energies", "pairs", "output", "inout", "trivial", "constraint"):
        mods[name] = __import__(name)
    return mods


def _setup(m, ref, case):
    cwd = os.getcwd()
    os.chdir(ref)      # forces.py reads _forces.yml relative to the working directory
    try:
        params = m["params"].init_params(imode=1, tfft=True, mprint=case.get("mprint", 1), nof=0)
        forces = m["forces"].init_forces(params, **case["force"])
    finally:
        os.chdir(cwd)
    grids = m["grids"].init_grids(params, **case["grid"])
    dens = m["densities"].init_densities(grids)
    mf = m["meanfield"].init_meanfield(grids)
    levels = m["levels"].init_levels(grids, **case["levels"])
    forces, static = m["static"].init_static(forces, levels, **case["static"])
    coul = m["coulomb"].init_coulomb(grids)
    en = m["energies"].init_energies()
    moment = m["moment"].init_moment(np.array([0.0, 0.0, 0.0]))
    pairs = m["pairs"].Pairs()
    return params, forces, grids, dens, mf, levels, static, coul, en, moment, pairs


def run_case(m, ref, name, case):
    params, forces, grids, dens, mf, levels, static, coul, en, moment, pairs = _setup(m, ref, case)
    levels = m["static"].harmosc(grids, levels, params, static)
    psi0 = np.array(levels.psi)
    hist = []
    st_mod = m["static"]
    orig_sum = st_mod.sum_energy

    def recording_sum_energy(energies, lv, meanfield, pr):
        e = orig_sum(energies, lv, meanfield, pr)
        hist.append((params.iteration, float(e.ehf), float(e.ehfint), float(e.efluct1[0]), float(e.efluct2[0]),
                     float(static.x0dmp), float(np.sum(pr.epair))))
        return e

    st_mod.sum_energy = recording_sum_energy
    st_mod.lastdiag = lambda *a, **k: (np.zeros(0), np.zeros(0))   # post-loop printout only
    tmp = tempfile.mkdtemp()
    cwd = os.getcwd()
    os.chdir(tmp)
    try:
        with contextlib.redirect_stdout(io.StringIO()):
            out = st_mod.statichf_with_benchmark(coul, dens, en, forces, grids, levels, mf, moment, params,
                                                 static, pairs, m["output"].FortranOutputWriter(tmp))
    finally:
        os.chdir(cwd)
        st_mod.sum_energy = orig_sum
    coul, dens, en, forces, grids, levels, mf = out[:7]
    obs_mod = m["output"]
    with contextlib.redirect_stdout(io.StringIO()):
        obs = obs_mod.calculate_complete_observables(dens, levels, grids, params)
    h = np.array(hist)
    np.savez_compressed(
        os.path.join(HERE, f"run_{name}.npz"),
        hist_iter=h[:, 0], hist_ehf=h[:, 1], hist_ehfint=h[:, 2], hist_efluct1=h[:, 3],
        hist_efluct2=h[:, 4], hist_x0dmp=h[:, 5], hist_epair=h[:, 6],
        psi0=psi0,
        rho=np.asarray(dens.rho), tau=np.asarray(dens.tau), chi=np.asarray(dens.chi),
        sp_energy=np.asarray(levels.sp_energy), sp_kinetic=np.asarray(levels.sp_kinetic),
        wocc=np.asarray(levels.wocc), wguv=np.asarray(levels.wguv), pairwg=np.asarray(levels.pairwg),
        wstates=np.asarray(levels.wstates), deltaf=np.asarray(levels.deltaf),
        eferm=np.asarray(pairs.eferm), epair=np.asarray(pairs.epair),
        rms=np.asarray(obs.rms), rmstot=np.asarray(obs.rmstot),
        ehf=float(en.ehf), ehfint=float(en.ehfint),
        upot=np.asarray(mf.upot), wcoul=np.asarray(coul.wcoul))
    print(f"{name}: {len(hist)} energy records, ehf={en.ehf:.10f}")


def config_run(m, ref, name, workload, maxiter):
    """A bench workload (hfb.config preset) through the reference driver
    ``statichf_with_benchmark`` for ``maxiter`` iterations.  Records the
    per-iteration scalars, the final single-particle energies, occupations
    and radii, and the post-loop ``lastdiag`` of each isospin: its inputs
    (h and gap matrices, occupations, Fermi energies) and its quasiparticle
    energies and lower-component norms."""
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "jax-hfbfft_b200"))
    from hfb import config   # the workload presets (plain Python data; nothing is computed by hfb here)
    case = config.case_dict(workload, static=dict(maxiter=maxiter, iternat=0))
    params, forces, grids, dens, mf, levels, static, coul, en, moment, pairs = _setup(m, ref, case)
    levels = m["static"].harmosc(grids, levels, params, static)
    hist = []
    st_mod = m["static"]
    orig_sum, orig_last = st_mod.sum_energy, st_mod.lastdiag
    lastd = {}

    def recording_sum_energy(energies, lv, meanfield, pr):
        e = orig_sum(energies, lv, meanfield, pr)
        hist.append((params.iteration, float(e.ehf), float(e.ehfint), float(e.efluct1[0]), float(e.efluct2[0]),
                     float(static.x0dmp), float(np.sum(pr.epair))))
        return e

    def recording_lastdiag(f, g, lv, pa, stc, pr, iq):
        if iq == 0:
            lastd["hmatrix"] = np.array(stc.hmatrix)
            lastd["gapmatrix"] = np.array(stc.gapmatrix)
            lastd["wocc"] = np.array(lv.wocc)
            lastd["eferm"] = np.array(pr.eferm)
        qe, qn = orig_last(f, g, lv, pa, stc, pr, iq)
        lastd[f"qp_energy_{iq}"], lastd[f"qp_norm_{iq}"] = np.asarray(qe), np.asarray(qn)
        return qe, qn

    st_mod.sum_energy = recording_sum_energy
    st_mod.lastdiag = recording_lastdiag
    tmp = tempfile.mkdtemp()
    cwd = os.getcwd()
    os.chdir(tmp)
    try:
        with contextlib.redirect_stdout(io.StringIO()):
            out = st_mod.statichf_with_benchmark(coul, dens, en, forces, grids, levels, mf, moment, params,
                                                 static, pairs, m["output"].FortranOutputWriter(tmp))
    finally:
        os.chdir(cwd)
        st_mod.sum_energy, st_mod.lastdiag = orig_sum, orig_last
    coul, dens, en, forces, grids, levels, mf = out[:7]
    with contextlib.redirect_stdout(io.StringIO()):
        obs = m["output"].calculate_complete_observables(dens, levels, grids, params)
    h = np.array(hist)
    extra = {}
    if grids.nx <= 24:       # small enough to keep the final densities
        extra = dict(rho=np.asarray(dens.rho), tau=np.asarray(dens.tau))
    np.savez_compressed(
        os.path.join(HERE, f"config_{name}.npz"),
        workload=workload, maxiter=maxiter,
        hist_iter=h[:, 0], hist_ehf=h[:, 1], hist_ehfint=h[:, 2], hist_efluct1=h[:, 3],
        hist_efluct2=h[:, 4], hist_x0dmp=h[:, 5], hist_epair=h[:, 6],
        sp_energy=np.asarray(levels.sp_energy), sp_kinetic=np.asarray(levels.sp_kinetic),
        sp_norm=np.asarray(levels.sp_norm),
        wocc=np.asarray(levels.wocc), wguv=np.asarray(levels.wguv), deltaf=np.asarray(levels.deltaf),
        eferm=np.asarray(pairs.eferm), epair=np.asarray(pairs.epair),
        rms=np.asarray(obs.rms), rmstot=np.asarray(obs.rmstot),
        ehf=float(en.ehf), ehfint=float(en.ehfint),
        nneut=levels.nneut, nprot=levels.nprot, npsi=np.asarray(levels.npsi),
        **{f"lastdiag_{k}": v for k, v in lastd.items()}, **extra)
    print(f"{name}: {len(hist)} energy records, ehf={en.ehf:.10f}", flush=True)


def natural_vectors(m, ref):
    """static.hfb_natural (configuration-space sub-iterations) on seeded
    inputs on an 8^3 grid (3 + 2 particles in 4 + 3 states): Hermitian h and
    gap matrices, an anti-Hermitian symcond, ascending single-particle
    energies and random occupation weights, three sub-iterations for each
    isospin in turn, once with state-dependent damping (e0bas = 10) and once
    with the global one (e0bas = 0).  Pairing is off (forces.ipair = 0): with
    it on, the reference's sub-iteration calls its single-isospin BCS solver
    with a missing argument (static.py:988)."""
    import jax.numpy as jnp
    J = jnp.asarray
    rng = np.random.default_rng(20261204)
    n = 8
    case = dict(grid=dict(nx=n, ny=n, nz=n, dx=0.9, dy=0.9, dz=0.9),
                force=dict(name="SLy4", ipair=0, tbcs=False),
                levels=dict(nneut=3, nprot=2, npsi=[4, 3]),
                static=dict(maxiter=1, radinx=2.0, radiny=2.1, radinz=2.4, serr=1e-20, x0dmp=0.3, e0dmp=100.0),
                mprint=1)
    out = {}
    for tag, e0bas in (("e0", 10.0), ("glob", 0.0)):
        params, forces, grids, dens, mf, levels, static, coul, en, moment, pairs = _setup(m, ref, case)
        nst, ld = levels.nstmax, max(levels.npsi)

        def herm(scale):
            a = rng.normal(size=(2, ld, ld)) + 1j * rng.normal(size=(2, ld, ld))
            return scale * 0.5 * (a + np.conj(np.transpose(a, (0, 2, 1))))

        h = herm(2.0)
        spe = np.concatenate([np.sort(rng.uniform(-40, 5, levels.npsi[0])), np.sort(rng.uniform(-35, 8, levels.npsi[1]))])
        for iq in range(2):
            off = 0 if iq == 0 else levels.npsi[0]
            for i in range(levels.npsi[iq]):
                h[iq, i, i] = spe[off + i]
        a = 0.3 * (rng.normal(size=(2, ld, ld)) + 1j * rng.normal(size=(2, ld, ld)))
        sym = 0.5 * (a - np.conj(np.transpose(a, (0, 2, 1))))
        ins = dict(psi=(rng.normal(size=(nst, 2, n, n, n)) + 1j * rng.normal(size=(nst, 2, n, n, n))) * 0.1,
                   lagrange=(rng.normal(size=(nst, 2, n, n, n)) + 1j * rng.normal(size=(nst, 2, n, n, n))) * 0.1,
                   hmatrix=h, gapmatrix=herm(0.5), symcond=sym, lambda_save=herm(1.0), sp_energy=spe,
                   wocc=rng.uniform(0.0, 1.0, nst), wguv=rng.uniform(0.0, 0.5, nst),
                   pairwg=rng.uniform(0.5, 1.0, nst), wstates=rng.uniform(0.8, 1.0, nst),
                   deltaf=rng.uniform(0.0, 2.0, nst))
        for k in ("psi", "lagrange", "sp_energy", "wocc", "wguv", "pairwg", "wstates", "deltaf"):
            setattr(levels, k, J(ins[k]))
        for k in ("hmatrix", "gapmatrix", "symcond", "lambda_save"):
            setattr(static, k, J(ins[k]))
        static.e0bas = e0bas
        static.delstepbas = 2.0
        for k, v in ins.items():
            out[f"{tag}_in_{k}"] = np.asarray(v)
        for iq in range(2):
            levels, static = m["static"].hfb_natural(forces, grids, levels, mf, params, static, iq, 3)
        for k in ("psi", "lagrange", "sp_energy", "deltaf"):
            out[f"{tag}_out_{k}"] = np.asarray(getattr(levels, k))
        for k in ("hmatrix", "gapmatrix", "symcond", "lambda_save"):
            out[f"{tag}_out_{k}"] = np.asarray(getattr(static, k))
    np.savez_compressed(os.path.join(HERE, "natural_n8.npz"), **out)
    print("natural_n8: hfb_natural on seeded inputs", flush=True)


def _smooth_random(rng, shape, n, scale):
    """Seeded smooth random field: a few low Fourier modes, real."""
    f = np.zeros(shape, dtype=np.complex128)
    lead = shape[:-3]
    for _ in range(6):
        k = rng.integers(-2, 3, size=3)
        amp = rng.normal(size=lead) + 1j * rng.normal(size=lead)
        ph = np.exp(2j * np.pi * (k[0] * np.arange(n)[:, None, None] + k[1] * np.arange(n)[None, :, None]
                                  + k[2] * np.arange(n)[None, None, :]) / n)
        f = f + np.asarray(amp)[..., None, None, None] * ph
    return scale * f.real


def unit_vectors(m, ref):
    """Per-function golden vectors on an 8^3 grid, dx=0.9, seeded inputs."""
    rng = np.random.default_rng(20261203)
    n = 8
    case = dict(grid=dict(nx=n, ny=n, nz=n, dx=0.9, dy=0.9, dz=0.9),
                force=dict(name="SLy4", ipair=6, tbcs=False, v0prot=362.0, v0neut=362.0, rho0pr=0.32),
                levels=dict(nneut=3, nprot=2, npsi=[4, 3]),
                static=dict(maxiter=1, radinx=2.0, radiny=2.1, radinz=2.4, serr=1e-20, x0dmp=0.3, e0dmp=100.0),
                mprint=1)
    params, forces, grids, dens, mf, levels, static, coul, en, moment, pairs = _setup(m, ref, case)
    import jax.numpy as jnp  # the stand-in: arrays assigned into reference objects need ``.at``
    J = jnp.asarray
    lev = m["levels"]
    out = {}
    psi = rng.normal(size=(2, n, n, n)) + 1j * rng.normal(size=(2, n, n, n))
    bfield = 20.0 + _smooth_random(rng, (n, n, n), n, 1.0)
    out["in_psi"] = psi
    out["in_b"] = bfield
    for ax, tag in ((1, "x"), (2, "y"), (3, "z")):
        out[f"cderv{tag}00"] = np.asarray(getattr(lev, f"cderv{tag}00")(0.9, psi))
        d1, d2 = getattr(lev, f"cderv{tag}01")(0.9, psi)
        out[f"cderv{tag}01_d1"], out[f"cderv{tag}01_d2"] = np.asarray(d1), np.asarray(d2)
        d1, d2 = getattr(lev, f"cderv{tag}02")(0.9, psi, bfield)
        out[f"cderv{tag}02_d1"], out[f"cderv{tag}02_d2"] = np.asarray(d1), np.asarray(d2)
    out["laplace_bcs"] = np.asarray(lev.laplace(0, 0, grids, forces, levels, 1.0, 0.0, psi, 0.0, 100.0))
    out["laplace_hfb"] = np.asarray(lev.laplace(0, 0, grids, forces, levels, 0.37, 0.02, psi, 3.5, 100.0))
    # hpsi01 with seeded smooth potentials
    s4 = (2, n, n, n)
    s5 = (2, 3, n, n, n)
    mf.upot = J(-50.0 + _smooth_random(rng, s4, n, 10.0))
    mf.bmass = J(20.0 + _smooth_random(rng, s4, n, 2.0))
    mf.v_pair = J(_smooth_random(rng, s4, n, 5.0))
    mf.aq = J(_smooth_random(rng, s5, n, 1.0))
    mf.spot = J(_smooth_random(rng, s5, n, 1.0))
    mf.wlspot = J(_smooth_random(rng, s5, n, 3.0))
    for k in ("upot", "bmass", "v_pair", "aq", "spot", "wlspot"):
        out[f"in_mf_{k}"] = np.asarray(getattr(mf, k))
    for iq in range(2):
        po, pm, pd = m["meanfield"].hpsi01(grids, mf, iq, 0.8, 0.3, psi)
        out[f"hpsi_iq{iq}_pout"], out[f"hpsi_iq{iq}_mf"], out[f"hpsi_iq{iq}_del"] = (
            np.asarray(po), np.asarray(pm), np.asarray(pd))
    # add_density on seeded states and weights
    nst = levels.nstmax
    levels.psi = J((rng.normal(size=(nst, 2, n, n, n)) + 1j * rng.normal(size=(nst, 2, n, n, n))) * 0.05)
    levels.wocc = J(rng.uniform(0.0, 1.0, size=nst))
    levels.wguv = J(rng.uniform(0.0, 0.5, size=nst))
    levels.pairwg = J(rng.uniform(0.5, 1.0, size=nst))
    levels.wstates = J(rng.uniform(0.8, 1.0, size=nst))
    out["in_dens_psi"] = np.asarray(levels.psi)
    for k in ("wocc", "wguv", "pairwg", "wstates"):
        out[f"in_dens_{k}"] = np.asarray(getattr(levels, k))
    d = m["densities"].add_density(dens, grids, levels)
    for k in ("rho", "chi", "tau", "current", "sdens", "sodens"):
        out[f"dens_{k}"] = np.asarray(getattr(d, k))
    # skyrme on physical-looking densities (Gaussian rho/tau/chi plus the seeded vector fields)
    x = np.asarray(grids.x)
    r2 = x[:, None, None] ** 2 + x[None, :, None] ** 2 + (1.1 * x[None, None, :]) ** 2
    d.rho = J(np.stack([0.08 * np.exp(-r2 / 6.0), 0.07 * np.exp(-r2 / 5.5)]))
    d.tau = J(np.stack([0.1 * np.exp(-r2 / 5.0), 0.09 * np.exp(-r2 / 5.0)]))
    d.chi = J(np.stack([0.01 * np.exp(-r2 / 7.0), 0.012 * np.exp(-r2 / 7.0)]))
    for k in ("rho", "tau", "chi"):
        out[f"in_sky_{k}"] = np.asarray(getattr(d, k))
    with contextlib.redirect_stdout(io.StringIO()):
        mf2, coul2 = m["meanfield"].skyrme(coul, d, forces, grids, mf, params, static)
    for k in ("upot", "bmass", "divaq", "v_pair", "aq", "spot", "wlspot", "dbmass"):
        out[f"sky_{k}"] = np.asarray(getattr(mf2, k))
    out["sky_ecorrp"] = float(mf2.ecorrp)
    out["sky_wcoul"] = np.asarray(coul2.wcoul)
    out["coulomb_q"] = np.asarray(coul2.q)
    # energies on the same densities and levels
    levels.sp_energy = J(rng.uniform(-40.0, 5.0, size=nst))
    levels.sp_kinetic = J(rng.uniform(5.0, 30.0, size=nst))
    pairs.epair = J(np.array([1.3, 0.7]))
    out["in_en_sp_energy"] = np.asarray(levels.sp_energy)
    out["in_en_sp_kinetic"] = np.asarray(levels.sp_kinetic)
    e = m["energies"].integ_energy(coul2, d, en, forces, grids, levels, params, pairs)
    e = m["energies"].sum_energy(e, levels, mf2, pairs)
    for k in ("ehft", "ehf0", "ehf1", "ehf2", "ehf3", "ehfls", "ehflsodd", "ehfc", "ecorc", "ehfint",
              "e3corr", "ehf", "tke", "ehfCrho0", "ehfCrho1", "ehfCdrho0", "ehfCdrho1", "ehfCtau0",
              "ehfCtau1", "ehfCdJ0", "ehfCdJ1"):
        out[f"en_{k}"] = float(getattr(e, k))
    # sp_properties
    lv = m["inout"].sp_properties(forces, grids, levels, moment)
    for k in ("sp_kinetic", "sp_spin", "sp_orbital", "sp_parity"):
        out[f"spp_{k}"] = np.asarray(getattr(lv, k))
    # BCS on synthetic spectra
    levels.sp_energy = J(np.sort(rng.uniform(-30.0, 10.0, size=nst)))
    levels.deltaf = J(rng.uniform(0.5, 2.0, size=nst))
    levels.wstates = J(np.ones(nst))
    levels.pairwg = J(np.ones(nst))
    out["in_bcs_sp_energy"] = np.asarray(levels.sp_energy)
    out["in_bcs_deltaf"] = np.asarray(levels.deltaf)
    params.iteration = 11
    forces.pair_cutoff = J(np.array([5.0, 5.0]))
    forces.state_cutoff = J(np.array([20.0, 20.0]))
    pr = m["pairs"].Pairs()
    pr.firstcall = False
    with contextlib.redirect_stdout(io.StringIO()):
        lv, pr = m["pairs"].pair(levels, mf2, forces, params, grids, pr)
    for k in ("wocc", "wguv", "pairwg", "wstates", "deltaf"):
        out[f"bcs_{k}"] = np.asarray(getattr(lv, k))
    for k in ("eferm", "epair", "avdelt", "avdeltv2", "avg"):
        out[f"bcs_{k}"] = np.asarray(getattr(pr, k))
    np.savez_compressed(os.path.join(HERE, "unit_n8.npz"), **out)
    print(f"unit_n8: {len(out)} arrays")


OBS_KEYS = ("pnr", "pnrtot", "cm", "cmtot", "dipole_isovector", "rms", "rmstot", "x2m", "x2mtot", "q20", "q22",
            "q20tot", "q22tot", "q20T1", "beta20tot", "beta22tot", "beta", "gamma", "pcm")


def observables_vectors(m, ref):
    """output.calculate_complete_observables on the final densities of the
    run fixtures (16^3) and on a seeded triaxial, off-centre density with
    currents; the density part of the observables (particle numbers, centres
    of mass, radii, second moments, quadrupole tensors, deformation,
    isovector dipole, summed currents)."""
    import types
    import jax.numpy as jnp
    out = {}
    items = [(name, case, np.load(os.path.join(HERE, f"run_{name}.npz"))["rho"], None)
             for name, case in RUN_CASES.items()]
    rng = np.random.default_rng(20261204)
    n = 16
    tri = dict(grid=dict(nx=n, ny=n, nz=n, dx=1.0, dy=1.1, dz=0.9), force=dict(name="SLy4", ipair=0, tbcs=False),
               levels=dict(nneut=12, nprot=10, npsi=[12, 10]),
               static=dict(maxiter=1, radinx=2.0, radiny=2.0, radinz=2.0, serr=1e-20, x0dmp=0.2, e0dmp=100.0),
               mprint=1)
    h = np.array([1.0, 1.1, 0.9])
    xs = [(np.arange(1, n + 1) - (n + 1) / 2) * h[d] for d in range(3)]
    X, Y, Z = np.meshgrid(*xs, indexing="ij")
    rho = np.stack([0.16 * np.exp(-((X - 0.4) / 3.1) ** 2 - ((Y + 0.3) / 2.6) ** 2 - ((Z - 0.2) / 3.8) ** 2),
                    0.15 * np.exp(-((X - 0.3) / 3.0) ** 2 - ((Y + 0.2) / 2.7) ** 2 - ((Z - 0.1) / 3.6) ** 2)])
    rho = rho * (1.0 + 0.05 * _smooth_random(rng, (2, n, n, n), n, 1.0))
    cur = _smooth_random(rng, (2, 3, n, n, n), n, 0.01) + 0.002 * rng.normal(size=(2, 3, 1, 1, 1))
    items.append(("triaxial_n16", tri, rho, cur))
    for name, case, rho, cur in items:
        params, forces, grids, dens, mf, levels, static, coul, en, moment, pairs = _setup(m, ref, case)
        d = types.SimpleNamespace(rho=jnp.asarray(rho))
        with contextlib.redirect_stdout(io.StringIO()):
            obs = m["output"].calculate_complete_observables(d, levels, grids, params,
                                                             None if cur is None else jnp.asarray(cur))
        out[f"{name}_rho"] = np.asarray(rho)
        if cur is not None:
            out[f"{name}_current"] = np.asarray(cur)
        out[f"{name}_grid"] = np.array([case["grid"]["nx"], case["grid"]["dx"], case["grid"]["dy"],
                                        case["grid"]["dz"]])
        out[f"{name}_nucleons"] = np.array([levels.nneut, levels.nprot], dtype=float)
        for k in OBS_KEYS:
            out[f"{name}_{k}"] = np.asarray(getattr(obs, k), dtype=float)
    np.savez_compressed(os.path.join(HERE, "observables_n16.npz"), **out)
    print(f"observables_n16: {len(items)} densities")


def res_writer_vectors(m, ref):
    """Text written by the reference's FortranOutputWriter (output.py:49-174)
    for three iterations of seeded synthetic energies, observables, damping
    and pairing values; the inputs are stored beside the file contents."""
    import json
    import types
    rng = np.random.default_rng(20261205)
    iters = []
    prev = 0.0
    for it in range(3):
        en = {k: float(rng.normal(0.0, 50.0)) for k in
              ("ehf", "ehfint", "tke", "ehfc", "ehfCrho0", "ehfCrho1", "ehfCdrho0", "ehfCdrho1", "ehfCtau0",
               "ehfCtau1", "ehfCdJ0", "ehfCdJ1", "e_zpe")}
        en["ehfprev"] = prev
        en["efluct1"] = [float(abs(rng.normal(0.0, 1e-3)))]
        en["efluct2"] = [float(abs(rng.normal(0.0, 1e-3)))]
        prev = en["ehf"]
        ob = dict(pnr=rng.uniform(5, 90, 2).tolist(), cmtot=rng.normal(0, 1e-3, 3).tolist(),
                  dipole_isovector=rng.normal(0, 1e-2, 3).tolist(), orbital_momentum=rng.normal(0, 1, 3).tolist(),
                  spin_momentum=rng.normal(0, 0.5, 3).tolist(), rms=rng.uniform(2, 6, 2).tolist(),
                  q20=rng.normal(0, 30, 2).tolist(), x2mtot=rng.uniform(1, 20, 3).tolist(),
                  pcm=rng.normal(0, 1e-2, (3, 2)).tolist())
        ob["total_momentum"] = (np.array(ob["orbital_momentum"]) + np.array(ob["spin_momentum"])).tolist()
        ob["pnrtot"] = ob["pnr"][0] + ob["pnr"][1]
        for k in ("rmstot", "q20tot", "q22tot", "beta"):
            ob[k] = float(abs(rng.normal(0, 3)))
        ob["gamma"] = float(rng.uniform(0, 60))
        iters.append(dict(iteration=it, energies=en, observables=ob, x0dmp=float(rng.uniform(0.1, 0.9)),
                          epair=rng.normal(-5, 2, 2).tolist()))
    tmp = tempfile.mkdtemp()
    w = m["output"].FortranOutputWriter(tmp)
    for d in iters:
        en = types.SimpleNamespace(**d["energies"])
        ob = types.SimpleNamespace(**{k: (np.array(v) if isinstance(v, list) else v)
                                      for k, v in d["observables"].items()})
        w.write_iteration_data(d["iteration"], en, ob, types.SimpleNamespace(x0dmp=d["x0dmp"]),
                               types.SimpleNamespace(epair=np.array(d["epair"])))
    files = {}
    for k, path in w.files.items():
        with open(path) as f:
            files[os.path.basename(path)] = f.read()
    with open(os.path.join(HERE, "res_files.json"), "w") as f:
        json.dump(dict(inputs=iters, files=files), f, indent=1)
    print(f"res_files: {len(files)} files")


def constraint_vectors(m, ref):
    """The reference's constraint module (constraint.py:47-342; not wired
    into its driver) on a 16^3 grid: the constraint fields for Q20 + Q22 +
    principal axes, expectation values and variances of a seeded density,
    one multiplier update, the wave-function correction of seeded states
    and the constraint potential."""
    import types
    import jax.numpy as jnp
    c = __import__("constraint")
    n = 16
    case = dict(grid=dict(nx=n, ny=n, nz=n, dx=1.0, dy=1.0, dz=1.0), force=dict(name="SLy4", ipair=0, tbcs=False),
                levels=dict(nneut=8, nprot=8, npsi=[5, 4]),
                static=dict(maxiter=1, radinx=2.0, radiny=2.0, radinz=2.0, serr=1e-20, x0dmp=0.2, e0dmp=100.0),
                mprint=1)
    params, forces, grids, dens, mf, levels, static, coul, en, moment, pairs = _setup(m, ref, case)
    rng = np.random.default_rng(20261206)
    with contextlib.redirect_stdout(io.StringIO()):
        cs = c.init_constraints(dict(alpha20_wanted=0.3, alpha22_wanted=0.05, tq_prin_axes=True), 16, grids)
    X, Y, Z = np.meshgrid(grids.x, grids.y, grids.z, indexing="ij")
    rho = np.stack([0.16 * np.exp(-(X / 2.8) ** 2 - (Y / 2.6) ** 2 - (Z / 3.3) ** 2),
                    0.15 * np.exp(-(X / 2.7) ** 2 - (Y / 2.6) ** 2 - (Z / 3.2) ** 2)])
    d = types.SimpleNamespace(rho=jnp.asarray(rho))
    ex, var = c.calculate_constraint_expectation_values(d, cs, grids)
    cs = cs.replace(old_crank=jnp.asarray(np.asarray(ex) * 0.9))
    cs2 = c.update_lagrange_multipliers(cs, ex, var, 100.0, 0.2)
    ns = 9
    psi = rng.normal(size=(ns, 2, n, n, n)) + 1j * rng.normal(size=(ns, 2, n, n, n))
    iso = np.array([1] * 5 + [2] * 4)
    wocc = rng.uniform(0.2, 1.0, ns)
    wst = np.ones(ns)
    lv = types.SimpleNamespace(isospin=jnp.asarray(iso), wocc=jnp.asarray(wocc), wstates=jnp.asarray(wst))
    # the reference's correction indexes fields [x, y, z, isospin] and
    # multiplies a spinor laid out [2, x, y, z] by [x, y, z, None]; it is
    # applied here to states stored [x, y, z, 2], the layout it indexes
    psi_xyzs = np.moveaxis(psi, 1, -1)
    cor = c.apply_wavefunction_corrections(jnp.asarray(psi_xyzs), cs2, lv)
    upot = rng.normal(size=(n, n, n, 2))
    pot = c.add_constraint_potential(jnp.asarray(upot), cs2)
    out = dict(rho=rho, fields=np.asarray(cs.constr_field), goals=np.asarray(cs.goal_crank),
               lambda0=np.asarray(cs.lambda_crank), old=np.asarray(cs.old_crank), expect=np.asarray(ex),
               var=np.asarray(var), lambda1=np.asarray(cs2.lambda_crank), qcorr=np.asarray(cs2.qcorr),
               psi=psi, isospin=iso, wocc=wocc, wstates=wst, psi_corrected=np.moveaxis(np.asarray(cor), -1, 1),
               upot_xyzs=upot, pot_xyzs=np.asarray(pot), mass_number=16.0)
    np.savez_compressed(os.path.join(HERE, "constraint_n16.npz"), **out)
    print(f"constraint_n16: {cs.numconstraint} constraints")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="path of the unmodified reference checkout")
    ap.add_argument("--only", default=None)
    a = ap.parse_args()
    m = _import_reference(a.ref)
    if a.only in (None, "unit"):
        unit_vectors(m, a.ref)
    if a.only in (None, "observables"):
        observables_vectors(m, a.ref)
    if a.only in (None, "res"):
        res_writer_vectors(m, a.ref)
    if a.only in (None, "constraint"):
        constraint_vectors(m, a.ref)
    if a.only in (None, "natural"):
        natural_vectors(m, a.ref)
    for name, case in RUN_CASES.items():
        if a.only in (None, name):
            m = _import_reference(a.ref)
            run_case(m, a.ref, name, case)
    for name, c in CONFIG_RUNS.items():
        if a.only in (None, "config", name):
            m = _import_reference(a.ref)
            config_run(m, a.ref, name, c["workload"], c["maxiter"])


if __name__ == "__main__":
    main()
