"""The oracle against golden vectors produced by the reference's own code.

Unit vectors (``unit_n8.npz``): every restated function on seeded inputs.
Run vectors (``run_*.npz``): the reference driver end to end on small grids;
the oracle must reproduce the per-iteration E_bind, the integrated EDF energy,
the rms of the antisymmetric lambda (efluct2), and the final densities,
levels and radii, with the reference's recorded step-size schedule replayed
(see ``oracle.static.iterate``).

``efluct1`` = max|lambda_asym| is compared loosely: it is not invariant under
unitary rotations inside degenerate (Kramers) subspaces, whose basis LAPACK
picks from rounding noise, so it is not reproducible between two correct
implementations.
"""
import copy
import os

import numpy as np
import pytest

from oracle import model, spectral, meanfield, densities, coulomb, pairs, energies, static
from cases import RUN_CASES

HERE = os.path.dirname(os.path.abspath(__file__))
G = os.path.join(HERE, "golden")


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def unit():
    return dict(np.load(os.path.join(G, "unit_n8.npz")))


def _unit_setup():
    g = model.init_grids(8, 8, 8, 0.9, 0.9, 0.9)
    f = model.init_forces("SLy4", ipair=6, tbcs=False, v0prot=362.0, v0neut=362.0, rho0pr=0.32)
    lv = model.init_levels(g, 3, 2, (4, 3))
    f, st = static.init_static(f, lv, maxiter=1, radinx=2.0, radiny=2.1, radinz=2.4, serr=1e-20,
                               x0dmp=0.3, e0dmp=100.0)
    return g, f, lv, st


def test_spectral_derivatives(unit):
    psi, b = unit["in_psi"], unit["in_b"]
    for ax, tag in ((1, "x"), (2, "y"), (3, "z")):
        assert rel(spectral.cderv00(0.9, psi, ax), unit[f"cderv{tag}00"]) < 1e-13
        d1, d2 = spectral.cderv01(0.9, psi, ax)
        assert rel(d1, unit[f"cderv{tag}01_d1"]) < 1e-13
        assert rel(d2, unit[f"cderv{tag}01_d2"]) < 1e-13
        d1, d2 = spectral.cderv02(0.9, psi, b, ax, ax - 1)
        assert rel(d1, unit[f"cderv{tag}02_d1"]) < 1e-13
        assert rel(d2, unit[f"cderv{tag}02_d2"]) < 1e-13


def test_laplace_preconditioner(unit):
    g, f, lv, st = _unit_setup()
    psi = unit["in_psi"]
    assert rel(spectral.laplace(g, f.h2ma, 1.0, 0.0, psi, 0.0, 100.0), unit["laplace_bcs"]) < 1e-13
    assert rel(spectral.laplace(g, f.h2ma, 0.37, 0.02, psi, 3.5, 100.0), unit["laplace_hfb"]) < 1e-13


def test_hpsi01(unit):
    g, f, lv, st = _unit_setup()
    mf = meanfield.init_meanfield(g)
    for k in ("upot", "bmass", "v_pair", "aq", "spot", "wlspot"):
        setattr(mf, k, unit[f"in_mf_{k}"])
    for iq in range(2):
        out = meanfield.hpsi01(g, mf, iq, 0.8, 0.3, unit["in_psi"])
        for o, tag in zip(out, ("pout", "mf", "del")):
            assert rel(o, unit[f"hpsi_iq{iq}_{tag}"]) < 1e-12, (iq, tag)


def test_hpsi01_matrix_form_equals_reference(unit):
    """The formulation of the single-precision tensor-core hpsi (a dense
    derivative GEMM per axis, the pointwise operator between two GEMMs and a
    rank-one Nyquist term) reproduces the reference's FFT-based hpsi01 in
    FP64 on its golden vectors (8^3, dx 0.9), and on a 16^3 grid with
    unequal spacings and smooth random fields against the oracle's
    FFT-based restatement."""
    g, f, lv, st = _unit_setup()
    mf = meanfield.init_meanfield(g)
    for k in ("upot", "bmass", "v_pair", "aq", "spot", "wlspot"):
        setattr(mf, k, unit[f"in_mf_{k}"])
    for iq in range(2):
        out = meanfield.hpsi01_matrix_form(g, mf, iq, 0.8, 0.3, unit["in_psi"])
        for o, tag in zip(out, ("pout", "mf", "del")):
            assert rel(o, unit[f"hpsi_iq{iq}_{tag}"]) < 1e-12, (iq, tag)
    rng = np.random.default_rng(16)
    n = 16
    g2 = model.init_grids(n, n, n, 0.8, 0.85, 0.9)
    x = np.arange(n)
    smooth = lambda: sum(rng.normal() * np.cos(2 * np.pi * (rng.integers(0, 3) * x[:, None, None]
                                                            + rng.integers(0, 3) * x[None, :, None]
                                                            + rng.integers(0, 3) * x[None, None, :]) / n
                                                   + rng.uniform(0, 6.3)) for _ in range(4))
    mf2 = meanfield.init_meanfield(g2)
    mf2.upot = np.stack([-40 + 5 * smooth(), -38 + 5 * smooth()])
    mf2.bmass = np.stack([20 + smooth(), 21 + smooth()])
    mf2.v_pair = np.stack([smooth(), smooth()])
    for k in ("aq", "spot", "wlspot"):
        setattr(mf2, k, np.stack([np.stack([0.3 * smooth() for _ in range(3)]) for _ in range(2)]))
    psi = rng.normal(size=(2, n, n, n)) + 1j * rng.normal(size=(2, n, n, n))
    for iq in range(2):
        a = meanfield.hpsi01(g2, mf2, iq, 0.7, 0.2, psi)
        b = meanfield.hpsi01_matrix_form(g2, mf2, iq, 0.7, 0.2, psi)
        for u, v in zip(a, b):
            assert rel(v, u) < 1e-12


def test_add_density(unit):
    g, f, lv, st = _unit_setup()
    lv.psi = unit["in_dens_psi"]
    for k in ("wocc", "wguv", "pairwg", "wstates"):
        setattr(lv, k, unit[f"in_dens_{k}"])
    d = densities.add_density(densities.init_densities(g), g, lv)
    for k in ("rho", "chi", "tau", "current", "sdens", "sodens"):
        assert rel(getattr(d, k), unit[f"dens_{k}"]) < 1e-12, k


def _sky(unit):
    g, f, lv, st = _unit_setup()
    d = densities.init_densities(g)
    for k in ("current", "sdens", "sodens"):
        setattr(d, k, unit[f"dens_{k}"])
    for k in ("rho", "tau", "chi"):
        setattr(d, k, unit[f"in_sky_{k}"])
    mf = meanfield.init_meanfield(g)
    c = coulomb.init_coulomb(g)
    mf, c = meanfield.skyrme(c, d, f, g, mf)
    return g, f, lv, d, mf, c


def test_coulomb_green_function(unit):
    g, f, lv, st = _unit_setup()
    assert rel(coulomb.init_coulomb(g).q, unit["coulomb_q"]) < 1e-13


def test_skyrme_potentials(unit):
    g, f, lv, d, mf, c = _sky(unit)
    for k in ("upot", "bmass", "divaq", "v_pair", "aq", "spot", "wlspot", "dbmass"):
        assert rel(getattr(mf, k), unit[f"sky_{k}"]) < 1e-12, k
    assert abs(mf.ecorrp - unit["sky_ecorrp"]) <= 1e-12 * abs(unit["sky_ecorrp"])
    assert rel(c.wcoul, unit["sky_wcoul"]) < 1e-12


def test_energies(unit):
    g, f, lv, d, mf, c = _sky(unit)
    lv.sp_energy = unit["in_en_sp_energy"]
    lv.sp_kinetic = unit["in_en_sp_kinetic"]
    for k in ("wocc", "wguv", "pairwg", "wstates"):
        setattr(lv, k, unit[f"in_dens_{k}"])
    pr = pairs.Pairs()
    pr.epair = np.array([1.3, 0.7])
    e = energies.integ_energy(c, d, energies.Energies(), f, g, lv, pr)
    e = energies.sum_energy(e, lv, mf, pr)
    for k in ("ehft", "ehf0", "ehf1", "ehf2", "ehf3", "ehfls", "ehflsodd", "ehfc", "ecorc", "ehfint",
              "e3corr", "ehf", "tke", "ehfCrho0", "ehfCrho1", "ehfCdrho0", "ehfCdrho1", "ehfCtau0",
              "ehfCtau1", "ehfCdJ0", "ehfCdJ1"):
        ref = float(unit[f"en_{k}"])
        assert abs(getattr(e, k) - ref) <= 1e-11 * max(abs(ref), 1.0), k


def test_sp_properties(unit):
    g, f, lv, st = _unit_setup()
    lv.psi = unit["in_dens_psi"]
    lv = energies.sp_properties(f, g, lv)
    for k in ("sp_kinetic", "sp_spin", "sp_orbital", "sp_parity"):
        assert rel(getattr(lv, k), unit[f"spp_{k}"]) < 1e-12, k


def test_bcs(unit):
    g, f, lv, st = _unit_setup()
    lv.sp_energy = unit["in_bcs_sp_energy"].copy()
    lv.deltaf = unit["in_bcs_deltaf"].copy()
    lv.wstates = np.ones(lv.nstmax)
    lv.pairwg = np.ones(lv.nstmax)
    f.pair_cutoff = np.array([5.0, 5.0])
    f.state_cutoff = np.array([20.0, 20.0])
    pr = pairs.Pairs()
    pr.firstcall = False
    lv, pr = pairs.pair(lv, meanfield.init_meanfield(g), f, 11, g, pr)
    for k in ("wocc", "wguv", "pairwg", "wstates", "deltaf"):
        assert rel(getattr(lv, k), unit[f"bcs_{k}"]) < 1e-12, k
    for k in ("eferm", "epair", "avdelt", "avdeltv2", "avg"):
        assert rel(getattr(pr, k), unit[f"bcs_{k}"]) < 1e-12, k


def _sorted_levels(v, npsi):
    return np.concatenate([np.sort(v[:npsi[0]]), np.sort(v[npsi[0]:])])


@pytest.mark.parametrize("name", sorted(RUN_CASES))
def test_run_matches_reference_driver(name):
    ref = dict(np.load(os.path.join(G, f"run_{name}.npz")))
    case = copy.deepcopy(RUN_CASES[name])
    rs = static.build(case)
    assert rel(rs.levels.psi, ref["psi0"]) < 1e-14
    recs = []

    def cb(r, i):
        recs.append((r.en.ehf, r.en.ehfint, r.en.efluct1[0], r.en.efluct2[0]))

    static.prepare(rs)
    pre = (rs.en.ehf, rs.en.ehfint)
    for i in range(1, rs.st.maxiter + 1):
        x0_used = rs.st.x0dmp
        done = static.iterate(rs, i, x0_schedule=ref["hist_x0dmp"])
        cb(rs, i)
        assert abs(x0_used - ref["hist_x0dmp"][i]) <= 1e-12 * x0_used, f"x0dmp schedule diverged at {i}"
        if done:
            break
    h = np.array(recs)
    assert abs(pre[0] - ref["hist_ehf"][0]) < 1e-9
    np.testing.assert_allclose(h[:, 0], ref["hist_ehf"][1:], rtol=0, atol=1e-8)
    np.testing.assert_allclose(h[:, 1], ref["hist_ehfint"][1:], rtol=0, atol=1e-8)
    np.testing.assert_allclose(h[:, 3], ref["hist_efluct2"][1:], rtol=1e-6, atol=1e-12)
    # efluct1 is basis dependent: check the invariant bounds rms <= max <= nst * rms and loose agreement
    nmax = max(case["levels"]["npsi"])
    assert np.all(h[:, 2] >= h[:, 3] * (1 - 1e-12)) and np.all(h[:, 2] <= nmax * h[:, 3])
    np.testing.assert_allclose(h[:, 2], ref["hist_efluct1"][1:], rtol=0.5, atol=1e-12)
    lv = rs.levels
    assert rel(rs.dens.rho, ref["rho"]) < 1e-9
    assert rel(rs.dens.tau, ref["tau"]) < 1e-9
    if case["force"]["ipair"] != 0:
        assert rel(rs.dens.chi, ref["chi"]) < 1e-8
        assert rel(rs.pairs.eferm, ref["eferm"]) < 1e-9
        assert rel(rs.pairs.epair, ref["epair"]) < 1e-8
        assert rel(_sorted_levels(lv.wocc, lv.npsi), _sorted_levels(ref["wocc"], lv.npsi)) < 1e-8
    assert rel(_sorted_levels(lv.sp_energy, lv.npsi), _sorted_levels(ref["sp_energy"], lv.npsi)) < 1e-9
    rms, rmstot = energies.rms_radii(rs.dens, rs.grids)
    assert np.max(np.abs(rms - ref["rms"])) < 1e-10
    assert abs(rs.en.ehf - ref["ehf"]) < 1e-8


OBS_CASES = ("o16_n16", "ne20_vdi_n16", "o18_dddi_n16", "triaxial_n16")


def obs_case(name):
    """(oracle grids, rho, current or None, nneut, nprot, reference values)
    of one density of tests/golden/observables_n16.npz."""
    z = np.load(os.path.join(G, "observables_n16.npz"))
    n, dx, dy, dz = z[f"{name}_grid"]
    g = model.init_grids(int(n), int(n), int(n), dx, dy, dz)
    cur = z[f"{name}_current"] if f"{name}_current" in z.files else None
    nn, nz = z[f"{name}_nucleons"]
    ref = {k[len(name) + 1:]: z[k] for k in z.files if k.startswith(name + "_")}
    return g, z[f"{name}_rho"], cur, nn, nz, ref


@pytest.mark.parametrize("name", OBS_CASES)
def test_observables_oracle_against_reference(name):
    """Moments, quadrupole deformation and dipole of the oracle against the
    reference's calculate_complete_observables (output.py:177-340) on the
    final densities of the golden runs and a triaxial density with currents.
    gamma is compared only where the shape is deformed (beta > 0.01): for a
    spherical density it is the angle of rounding noise."""
    g, rho, cur, nn, nz, ref = obs_case(name)
    o = energies.observables(rho, g, nn, nz, cur)
    for k in ("pnr", "pnrtot", "cm", "cmtot", "dipole_isovector", "rms", "rmstot", "x2m", "x2mtot", "pcm"):
        np.testing.assert_allclose(o[k], ref[k], rtol=1e-12, atol=1e-12, err_msg=k)
    qs = max(1.0, float(np.max(np.abs(ref["q20"]))))
    for k in ("q20", "q22", "q20tot", "q22tot"):
        np.testing.assert_allclose(o[k], ref[k], rtol=0, atol=1e-11 * qs, err_msg=k)
    for k in ("q20T1", "beta20tot", "beta22tot", "beta"):
        np.testing.assert_allclose(o[k], ref[k], rtol=0, atol=1e-12, err_msg=k)
    if ref["beta"] > 0.01:
        assert abs(o["gamma"] - ref["gamma"]) < 1e-9


def test_constraint_oracle_against_reference():
    """The constraint restatement (oracle/constraint.py) against the
    reference's constraint.py functions on seeded inputs: fields, moments,
    one multiplier update, the state correction and the potential."""
    from oracle import constraint as oc
    z = np.load(os.path.join(G, "constraint_n16.npz"))
    g = model.init_grids(16, 16, 16, 1.0, 1.0, 1.0)
    f, names = oc.constraint_fields(g, oc.Q20 | oc.Q22 | oc.PRINCIPAL, float(z["mass_number"]))
    assert names == ["q20", "q22", "xy", "xz", "yz", "x", "y", "z"]
    ref_f = np.moveaxis(z["fields"], -1, 1)              # [i][iq][x][y][z]
    np.testing.assert_allclose(f, ref_f[:, 0], rtol=0, atol=1e-15)
    np.testing.assert_array_equal(ref_f[:, 0], ref_f[:, 1])
    ex, var = oc.expectation_values(f, z["rho"], g.wxyz)
    np.testing.assert_allclose(ex, z["expect"], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(var, z["var"], rtol=1e-12, atol=1e-15)
    lam, qc = oc.update_multipliers(z["lambda0"], z["old"], z["goals"], z["expect"], z["var"], 100.0, 0.2)
    np.testing.assert_allclose(lam, z["lambda1"], rtol=1e-13)
    np.testing.assert_allclose(qc, z["qcorr"], rtol=1e-13, atol=1e-16)
    cor = oc.correct_states(z["psi"], f, z["qcorr"], z["isospin"] - 1, z["wocc"], z["wstates"])
    assert rel(cor, z["psi_corrected"]) < 1e-13
    pot = oc.constraint_potential(np.moveaxis(z["upot_xyzs"], -1, 0), f, z["lambda1"])
    assert rel(pot, np.moveaxis(z["pot_xyzs"], -1, 0)) < 1e-14


# ---- lastdiag on the bench workloads' final matrices --------------------
from cases import CONFIG_RUNS  # noqa: E402


def qp_cluster_norms(e, q, tol=1e-7):
    """Quasiparticle norms summed in quadrature over clusters of degenerate
    energies (Kramers pairs): the norm of one eigenvector depends on the
    basis the eigensolver picks inside a degenerate subspace, the cluster
    sum does not.  Returns (cluster energies, cluster norms^2)."""
    e = np.asarray(e)
    q = np.asarray(q)
    ce, cq = [], []
    i = 0
    while i < len(e):
        j = i + 1
        while j < len(e) and abs(e[j] - e[i]) <= tol * max(1.0, abs(e[i])):
            j += 1
        ce.append(e[i])
        cq.append(float(np.sum(q[i:j] ** 2)))
        i = j
    return np.array(ce), np.array(cq)


@pytest.mark.parametrize("name", sorted(CONFIG_RUNS))
def test_oracle_lastdiag_matches_reference(name):
    """The restated lastdiag (reference index ranges) on the h and gap
    matrices, occupations and Fermi energies the reference driver held at
    its end reproduces the reference's quasiparticle energies and the
    degenerate-cluster sums of its lower-component norms."""
    d = np.load(os.path.join(G, f"config_{name}.npz"))
    nneut, nprot = int(d["nneut"]), int(d["nprot"])
    for iq in range(2):
        nst = nneut if iq == 0 else nprot
        start = 0 if iq == 0 else nneut
        e, q = static.lastdiag_block(d["lastdiag_hmatrix"][iq, :nst, :nst], d["lastdiag_gapmatrix"][iq, :nst, :nst],
                                     d["lastdiag_wocc"][start:start + nst], float(d["lastdiag_eferm"][iq]), start)
        er, qr = d[f"lastdiag_qp_energy_{iq}"], d[f"lastdiag_qp_norm_{iq}"]
        assert np.max(np.abs(e - er)) <= 1e-10 * max(1.0, np.max(np.abs(er)))
        ce, cq = qp_cluster_norms(e, q)
        cer, cqr = qp_cluster_norms(er, qr)
        assert len(ce) == len(cer)
        assert np.max(np.abs(cq - cqr)) <= 1e-10


# ---- hfb_natural on seeded inputs ---------------------------------------
@pytest.mark.parametrize("tag", ["e0", "glob"])
def test_oracle_hfb_natural_matches_reference(tag):
    """The restated configuration-space sub-iterations (reference index
    ranges, pairing off) reproduce the reference's hfb_natural: rotated
    states and Lagrange fields, transformed h and gap matrices, lambda,
    the updated symcond and single-particle energies."""
    import types
    d = np.load(os.path.join(G, "natural_n8.npz"))
    lv = types.SimpleNamespace(nneut=3, nprot=2, npsi=[4, 3], nstmax=7)
    for k in ("psi", "lagrange", "sp_energy", "wocc", "wguv", "pairwg", "wstates", "deltaf"):
        setattr(lv, k, d[f"{tag}_in_{k}"].copy())
    st = types.SimpleNamespace(e0bas=10.0 if tag == "e0" else 0.0, delstepbas=2.0)
    for k in ("hmatrix", "gapmatrix", "symcond", "lambda_save"):
        setattr(st, k, d[f"{tag}_in_{k}"].copy())
    for iq in range(2):
        static.hfb_natural(lv, st, iq, 3, reference_indexing=True)
    for k in ("psi", "lagrange", "sp_energy"):
        assert rel(getattr(lv, k), d[f"{tag}_out_{k}"]) < 1e-12, k
    for k in ("hmatrix", "gapmatrix", "symcond", "lambda_save"):
        assert rel(getattr(st, k), d[f"{tag}_out_{k}"]) < 1e-12, k
