"""CUDA kernels through the C ABI against the reference's golden vectors and
the oracle.  Tolerances: FP64 paths 1e-11 relative (max |diff| / max |ref|);
FP32 paths 3e-5 relative."""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from conftest import GOLDEN  # noqa: E402

TOL64 = 1e-11
TOL32 = 3e-5


def rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    b = b.detach().cpu().numpy() if isinstance(b, torch.Tensor) else np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def T(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return t.to(dtype) if dtype is not None else t


@pytest.fixture(scope="module")
def unit():
    return dict(np.load(os.path.join(GOLDEN, "unit_n8.npz")))


@pytest.fixture(scope="module")
def g8():
    import hfb
    from hfb import levels
    p = hfb.params.init_params()
    g = hfb.grids.init_grids(p, nx=8, ny=8, nz=8, dx=0.9, dy=0.9, dz=0.9)
    levels.use_grid(g)
    return g


def _forces8():
    import hfb
    f = hfb.forces.init_forces(None, name="SLy4", ipair=6, tbcs=False, v0prot=362.0, v0neut=362.0, rho0pr=0.32)
    a = 5   # the golden unit case has nneut = 3, nprot = 2 (h2m scaled by (A-1)/A)
    f.h2m = [h * (a - 1.0) / a for h in f.h2m]
    return f


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
def test_cderv_against_reference(unit, g8, dtype):
    from hfb import levels as L
    tol = TOL64 if dtype == torch.complex128 else TOL32
    psi = T(unit["in_psi"], dtype)
    b = T(unit["in_b"])
    for tag in ("x", "y", "z"):
        assert rel(getattr(L, f"cderv{tag}00")(0.9, psi), unit[f"cderv{tag}00"]) < tol
        d1, d2 = getattr(L, f"cderv{tag}01")(0.9, psi)
        assert rel(d1, unit[f"cderv{tag}01_d1"]) < tol and rel(d2, unit[f"cderv{tag}01_d2"]) < tol
        d1, d2 = getattr(L, f"cderv{tag}02")(0.9, psi, b)
        assert rel(d1, unit[f"cderv{tag}02_d1"]) < tol and rel(d2, unit[f"cderv{tag}02_d2"]) < tol, tag


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
def test_laplace_against_reference(unit, g8, dtype):
    from hfb import levels as L
    tol = TOL64 if dtype == torch.complex128 else TOL32
    f = _forces8()
    psi = T(unit["in_psi"], dtype)
    assert rel(L.laplace(0, 0, g8, f, None, 1.0, 0.0, psi, 0.0, 100.0), unit["laplace_bcs"]) < tol
    assert rel(L.laplace(0, 0, g8, f, None, 0.37, 0.02, psi, 3.5, 100.0), unit["laplace_hfb"]) < tol


def _mf_from_unit(g, unit, dtype):
    import hfb
    mf = hfb.meanfield.init_meanfield(g, dtype)
    for k in ("upot", "bmass", "v_pair", "aq", "spot", "wlspot"):
        getattr(mf, k).copy_(T(unit[f"in_mf_{k}"]))
    mf.pack(dtype)
    return mf


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
def test_hpsi01_against_reference(unit, g8, dtype):
    import hfb
    tol = TOL64 if dtype == torch.complex128 else 1e-4
    mf = _mf_from_unit(g8, unit, dtype)
    psi = T(unit["in_psi"], dtype)
    for iq in range(2):
        out = hfb.meanfield.hpsi01(g8, mf, iq, 0.8, 0.3, psi)
        for o, tag in zip(out, ("pout", "mf", "del")):
            assert rel(o, unit[f"hpsi_iq{iq}_{tag}"]) < tol, (iq, tag)


@pytest.mark.parametrize("n,dtype,ns", [(16, torch.complex128, 5), (24, torch.complex128, 5),
                                        (32, torch.complex64, 5), (48, torch.complex128, 5),
                                        (48, torch.complex64, 5), (40, torch.complex128, 5),
                                        (24, torch.complex64, 37), (40, torch.complex64, 6)])
def test_hpsi_batched_against_oracle(n, dtype, ns):
    """Batched hpsi over states of both isospins on larger grids vs the oracle
    (single precision on 24-48 grids runs the tensor-core kernel; 37 states on
    24^3 span several scheduling groups, the last one partial)."""
    _check_hpsi_batched(n, dtype, ns)


@pytest.mark.parametrize("n,ns", [(8, 3), (16, 5), (24, 5), (40, 5), (48, 5), (48, 9)])
def test_hpsi_fp64_fft_kernels_against_oracle(monkeypatch, n, ns):
    """FP64 hpsi by the FFT kernels (HFB_F64_HPSI=fft at context creation;
    the default is the FP64 tensor-core form, D as an n x n matrix and
    mma.sync m8n8k4 .f64, which the batched test above checks) against the
    oracle, to the same 1e-11."""
    monkeypatch.setenv("HFB_F64_HPSI", "fft")
    _check_hpsi_batched(n, torch.complex128, ns)


def _check_hpsi_batched(n, dtype, ns):
    import hfb
    from oracle import model, meanfield as omf
    rng = np.random.default_rng(n)
    d = (0.8, 0.85, 0.9)
    g = model.init_grids(n, n, n, *d)
    x = [(np.arange(n) - (n - 1) / 2) * h for h in d]
    r2 = x[0][:, None, None] ** 2 + x[1][None, :, None] ** 2 + x[2][None, None, :] ** 2
    w = np.exp(-r2 / (0.05 * (n * d[0]) ** 2))
    mfo = omf.init_meanfield(g)
    mfo.upot = np.stack([-50 * w, -45 * w])
    mfo.bmass = np.stack([20 + 2 * w, 21 + 1.5 * w])
    mfo.v_pair = np.stack([-3 * w, -2 * w])
    for k, s in (("aq", 0.3), ("spot", 0.2), ("wlspot", 1.0)):
        setattr(mfo, k, s * rng.standard_normal((2, 3, 1, 1, 1)) * w[None, None])
    nn = 3 if ns == 5 else ns // 2
    psi = (rng.standard_normal((ns, 2, n, n, n)) + 1j * rng.standard_normal((ns, 2, n, n, n))) * w
    wt = rng.uniform(0.2, 1.0, ns)
    wu = rng.uniform(0.0, 0.5, ns)
    p = hfb.params.init_params()
    gg = hfb.grids.init_grids(p, nx=n, ny=n, nz=n, dx=d[0], dy=d[1], dz=d[2])
    mf = hfb.meanfield.init_meanfield(gg, dtype)
    for k in ("upot", "bmass", "v_pair", "aq", "spot", "wlspot"):
        getattr(mf, k).copy_(T(getattr(mfo, k)))
    mf.pack(dtype)
    pt = T(psi, dtype)
    out = torch.empty_like(pt)
    omf_ = torch.empty_like(pt)
    odel = torch.empty_like(pt)
    wt_t, wu_t = T(wt), T(wu)          # keep the weight buffers alive across the launch
    from hfb._lib import call, ptr, stream_ptr, prec_of
    call("hfb_hpsi", gg.ctx.handle, prec_of(pt), ptr(mf.pot), ns, nn, ptr(pt), ptr(wt_t), ptr(wu_t), ptr(out),
         ptr(omf_), ptr(odel), stream_ptr())
    gg.ctx.check("hpsi")
    tol = 1e-11 if dtype == torch.complex128 else 1e-4
    for iq, sl in ((0, slice(0, nn)), (1, slice(nn, ns))):
        r = omf.hpsi01(g, mfo, iq, wt[sl], wu[sl], psi[sl])
        assert rel(out[sl], r[0]) < tol
        assert rel(omf_[sl], r[1]) < tol
        assert rel(odel[sl], r[2]) < tol


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
def test_add_density_against_reference(unit, g8, dtype):
    import hfb
    tol = TOL64 if dtype == torch.complex128 else 1e-5
    lv = hfb.levels.init_levels(g8, 3, 2, (4, 3), dtype=dtype)
    lv.psi.copy_(T(unit["in_dens_psi"], dtype))
    for k in ("wocc", "wguv", "pairwg", "wstates"):
        getattr(lv, k).copy_(T(unit[f"in_dens_{k}"]))
    d = hfb.densities.init_densities(g8)
    hfb.densities.add_density(d, g8, lv)
    for k in ("rho", "chi", "tau", "current", "sdens", "sodens"):
        assert rel(getattr(d, k), unit[f"dens_{k}"]) < tol, k


def test_kinetic_energy_against_reference(unit, g8):
    import hfb
    f = _forces8()
    lv = hfb.levels.init_levels(g8, 3, 2, (4, 3))
    lv.psi.copy_(T(unit["in_dens_psi"]))
    hfb.inout.sp_properties(f, g8, lv)
    assert rel(lv.sp_kinetic, unit["spp_sp_kinetic"]) < TOL64
    # orbital angular momentum, spin, parity (hfb_sp_properties)
    for k in ("sp_orbital", "sp_spin", "sp_parity"):
        assert rel(getattr(lv, k), unit[f"spp_{k}"]) < 1e-12, k
    lv32 = hfb.levels.init_levels(g8, 3, 2, (4, 3), dtype=torch.complex64)
    lv32.psi.copy_(T(unit["in_dens_psi"], torch.complex64))
    hfb.inout.sp_properties(f, g8, lv32)
    for k in ("sp_orbital", "sp_spin", "sp_parity"):
        assert rel(getattr(lv32, k), unit[f"spp_{k}"]) < 1e-5, k
    # the fused path inside add_density gives the same numbers
    for k in ("wocc", "wguv", "pairwg", "wstates"):
        getattr(lv, k).copy_(T(unit[f"in_dens_{k}"]))
    lv.sp_kinetic.zero_()
    hfb.densities.add_density(hfb.densities.init_densities(g8), g8, lv, forces=f)
    assert rel(lv.sp_kinetic, unit["spp_sp_kinetic"]) < TOL64


def _dens_for_skyrme(g8, unit):
    import hfb
    d = hfb.densities.init_densities(g8)
    for k in ("current", "sdens", "sodens"):
        getattr(d, k).copy_(T(unit[f"dens_{k}"]))
    for k in ("rho", "tau", "chi"):
        getattr(d, k).copy_(T(unit[f"in_sky_{k}"]))
    return d


def test_skyrme_and_coulomb_against_reference(unit, g8):
    import hfb
    f = _forces8()
    d = _dens_for_skyrme(g8, unit)
    mf = hfb.meanfield.init_meanfield(g8)
    c = hfb.coulomb.init_coulomb(g8)
    st = type("S", (), {"outertype": "N"})()
    hfb.meanfield.skyrme(c, d, f, g8, mf, hfb.params.init_params(), st)
    for k in ("upot", "bmass", "divaq", "v_pair", "aq", "spot", "wlspot", "dbmass"):
        assert rel(getattr(mf, k), unit[f"sky_{k}"]) < TOL64, k
    assert abs(mf.ecorrp - float(unit["sky_ecorrp"])) <= 1e-11 * abs(float(unit["sky_ecorrp"]))
    assert rel(c.wcoul, unit["sky_wcoul"]) < TOL64
    w = hfb.coulomb.poisson(g8, None, c, d.rho)
    assert rel(w, unit["sky_wcoul"]) < TOL64


def test_energies_against_reference(unit, g8):
    import hfb
    f = _forces8()
    d = _dens_for_skyrme(g8, unit)
    mf = hfb.meanfield.init_meanfield(g8)
    c = hfb.coulomb.init_coulomb(g8)
    st = type("S", (), {"outertype": "N"})()
    p = hfb.params.init_params()
    hfb.meanfield.skyrme(c, d, f, g8, mf, p, st)
    lv = hfb.levels.init_levels(g8, 3, 2, (4, 3))
    lv.sp_energy.copy_(T(unit["in_en_sp_energy"]))
    lv.sp_kinetic.copy_(T(unit["in_en_sp_kinetic"]))
    for k in ("wocc", "wguv", "pairwg", "wstates"):
        getattr(lv, k).copy_(T(unit[f"in_dens_{k}"]))
    pr = hfb.pairs.Pairs()
    pr.out[1] = torch.tensor([1.3, 0.7], dtype=torch.float64)
    e = hfb.energies.init_energies()
    hfb.energies.integ_energy(c, d, e, f, g8, lv, p, pr)
    hfb.energies.sum_energy(e, lv, mf, pr, grids=g8)
    e.sync()
    for k in ("ehft", "ehf0", "ehf1", "ehf2", "ehf3", "ehfls", "ehflsodd", "ehfc", "ecorc", "ehfint", "e3corr",
              "ehf", "tke", "ehfCrho0", "ehfCrho1", "ehfCdrho0", "ehfCdrho1", "ehfCtau0", "ehfCtau1", "ehfCdJ0",
              "ehfCdJ1"):
        ref = float(unit[f"en_{k}"])
        assert abs(getattr(e, k) - ref) <= 1e-10 * max(abs(ref), 1.0), (k, getattr(e, k), ref)


def test_bcs_against_reference(unit, g8):
    import hfb
    f = _forces8()
    f.pair_cutoff = (5.0, 5.0)
    f.state_cutoff = (20.0, 20.0)
    lv = hfb.levels.init_levels(g8, 3, 2, (4, 3))
    lv.sp_energy.copy_(T(unit["in_bcs_sp_energy"]))
    lv.deltaf.copy_(T(unit["in_bcs_deltaf"]))
    p = hfb.params.init_params()
    p.iteration = 11
    pr = hfb.pairs.Pairs()
    pr.firstcall = False
    hfb.pairs.pair(lv, None, f, p, g8, pr)
    g8.ctx.check("pair")
    for k in ("wocc", "wguv", "pairwg", "wstates", "deltaf"):
        assert rel(getattr(lv, k), unit[f"bcs_{k}"]) < 1e-12, k
    for k in ("eferm", "epair", "avdelt", "avdeltv2", "avg"):
        assert rel(getattr(pr, k), unit[f"bcs_{k}"]) < 1e-12, k


def test_bcs_not_bracketed_reports_status(g8):
    """A particle number that no Fermi level on [-100, 100] reaches latches
    HFB_ERR_NOT_BRACKETED (the reference's brentq raises)."""
    import hfb
    from hfb._lib import HfbError
    f = _forces8()
    lv = hfb.levels.init_levels(g8, 9, 2, (4, 3))       # 9 neutrons in 4 states
    p = hfb.params.init_params()
    p.iteration = 1
    hfb.pairs.pair(lv, None, f, p, g8, hfb.pairs.Pairs())
    with pytest.raises(HfbError) as e:
        g8.ctx.check("pair")
    assert e.value.code == 4


@pytest.mark.parametrize("n", [7, 40, 96, 140])
def test_eigh_jacobi(g8, n):
    import hfb
    from hfb._lib import call, ptr, stream_ptr
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    a = a + a.conj().T
    a[np.triu_indices(n, 1)] = 7.0 + 3.0j      # only the lower triangle may be read
    al = np.tril(a) + np.tril(a, -1).conj().T
    wref = np.linalg.eigvalsh(al)
    at = T(a.astype(np.complex128))
    w = torch.empty(n, dtype=torch.float64, device="cuda")
    v = torch.empty((n, n), dtype=torch.complex128, device="cuda")
    sw = torch.zeros(1, dtype=torch.int32, device="cuda")
    call("hfb_eigh", g8.ctx.handle, 1, n, n, ptr(at), ptr(w), ptr(v), ptr(sw), stream_ptr())
    g8.ctx.check("eigh")
    assert 1 <= int(sw[0]) <= 15, int(sw[0])
    wn, vn = w.cpu().numpy(), v.cpu().numpy()
    assert np.max(np.abs(wn - wref)) < 1e-11 * np.max(np.abs(wref))
    assert np.max(np.abs(vn.conj().T @ vn - np.eye(n))) < 1e-12
    assert np.max(np.abs(vn.conj().T @ al @ vn - np.diag(wn))) < 1e-11 * np.max(np.abs(wref))


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
def test_gram(dtype):
    import hfb
    from hfb._lib import call, ptr, stream_ptr, prec_of
    n = 16
    p = hfb.params.init_params()
    g = hfb.grids.init_grids(p, nx=n, ny=n, nz=n, dx=1.0, dy=1.0, dz=1.0)
    rng = np.random.default_rng(3)
    ns = 37
    K = 2 * n ** 3
    a = rng.standard_normal((3, ns, K)) + 1j * rng.standard_normal((3, ns, K))
    # the h psi slot holds a Hermitian operator applied to psi (here a real
    # diagonal one), so its Gram matrix is Hermitian as in the iteration
    a[2] = a[0] * rng.uniform(-2.0, 2.0, K)[None]
    vp = rng.standard_normal(n ** 3)
    out = torch.zeros((4, ns, ns), dtype=torch.complex128, device="cuda")
    ta = [T(x, dtype) for x in a]
    vpt = T(vp)
    call("hfb_gram", g.ctx.handle, prec_of(ta[0]), 0, ns, 15, ptr(ta[0]), ptr(ta[1]), ptr(ta[2]), ptr(vpt), 0.5,
         ptr(out), stream_ptr())
    x3 = a[0] * np.tile(vp, 2)[None]
    torch.cuda.synchronize()
    refs = [0.5 * a[0].conj() @ x.T for x in (a[0], a[1], a[2], x3)]
    tol = 1e-12 if dtype == torch.complex128 else 2e-5
    for k in range(4):
        assert rel(out[k], refs[k]) < tol, k


def _gram_case(n, s0, ns, seed):
    import hfb
    p = hfb.params.init_params()
    g = hfb.grids.init_grids(p, nx=n, ny=n, nz=n, dx=1.0, dy=1.0, dz=1.0)
    rng = np.random.default_rng(seed)
    K = 2 * n ** 3
    a = rng.standard_normal((3, s0 + ns, K)) + 1j * rng.standard_normal((3, s0 + ns, K))
    a[2] = a[0] * rng.uniform(-2.0, 2.0, K)[None]
    a = a.astype(np.complex64).astype(np.complex128)      # exact single-precision inputs
    vp = rng.standard_normal(n ** 3).astype(np.float32).astype(np.float64)
    return g, a, vp


def _gram_run(g, a, vp, s0, ns, dtype):
    from hfb._lib import call, ptr, stream_ptr, prec_of
    out = torch.zeros((4, ns, ns), dtype=torch.complex128, device="cuda")
    ta = [T(x, dtype) for x in a]
    vpt = T(vp)
    call("hfb_gram", g.ctx.handle, prec_of(ta[0]), s0, ns, 15, ptr(ta[0]), ptr(ta[1]), ptr(ta[2]), ptr(vpt), 0.5,
         ptr(out), stream_ptr())
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("n,s0,ns", [(16, 0, 140), (16, 5, 96), (16, 3, 9), (24, 0, 70)])
def test_gram_tensor_cores(n, s0, ns):
    """Single-precision Gram on tcgen05 (three-term tf32, windowed fp32
    accumulation, fp64 slice sums) against the fp64 Gram of the same
    single-precision inputs: max error below 3e-6 of max |C|; the Hermitian
    matrices' off-diagonal elements mirror exactly."""
    g, a, vp = _gram_case(n, s0, ns, 11)
    out = _gram_run(g, a, vp, s0, ns, torch.complex64)
    sl = slice(s0, s0 + ns)
    x3 = a[0][sl] * np.tile(vp, 2)[None]
    refs = [0.5 * a[0][sl].conj() @ x.T for x in (a[0][sl], a[1][sl], a[2][sl], x3)]
    for k in range(4):
        assert rel(out[k], refs[k]) < 3e-6, (k, rel(out[k], refs[k]))
    for k in (0, 2, 3):       # off-diagonal elements mirrored exactly
        assert np.array_equal(np.triu(out[k], 1), np.triu(out[k].conj().T, 1)), k


@pytest.mark.gpu
def test_gram_tensor_cores_match_cuda_cores(monkeypatch):
    """HFB_NO_TCGEN05=1 at context creation selects the CUDA-core kernel;
    both single-precision paths agree to single-precision accuracy."""
    n, s0, ns = 16, 2, 50
    g, a, vp = _gram_case(n, s0, ns, 12)
    tc = _gram_run(g, a, vp, s0, ns, torch.complex64)
    monkeypatch.setenv("HFB_NO_TCGEN05", "1")
    g2, _, _ = _gram_case(n, s0, ns, 12)
    cc = _gram_run(g2, a, vp, s0, ns, torch.complex64)
    for k in range(4):
        assert rel(tc[k], cc[k]) < 1e-5, k
        assert not np.array_equal(tc[k], cc[k]), k       # two different kernels ran


@pytest.mark.gpu
def test_diagstep_single_precision_matches_double():
    """hfb_diagstep on complex64 states (tensor-core Gram, Newton-Schulz
    S^-1/2, register-tiled rotation) against the same step on the complex128
    states it was rounded from, on Pb208 after two iterations (three 128-row
    Gram blocks, three rotation column tiles).  Gauge-invariant checks: every
    single-precision state lies in the span of the double-precision ones
    (row norms of the overlap matrix), and the single-particle energies
    agree."""
    import hfb
    from hfb import config, static
    sts = []
    for _ in range(2):
        st = config.setup(config.case_dict("Pb208"), dtype=torch.complex128)
        S = {k: st[k] for k in static._STATE_KEYS}
        static.prepare(**S)
        for i in (1, 2):
            static.iterate(i, **S)
        sts.append(st)
    static.to_precision(sts[1], torch.complex64)
    for st in sts:
        static.diagstep(st["energies"], st["forces"], st["grids"], st["levels"], st["static"], True, True)
    torch.cuda.synchronize()
    l64, l32 = sts[0]["levels"], sts[1]["levels"]
    wxyz = sts[0]["grids"].wxyz
    n0 = l64.npsi[0]
    for sl in (slice(0, n0), slice(n0, l64.nstmax)):
        a = l32.psi[sl].reshape(sl.stop - sl.start, -1).to(torch.complex128)
        b = l64.psi[sl].reshape(sl.stop - sl.start, -1)
        o = (a.conj() @ b.T) * wxyz
        rows = (o.abs() ** 2).sum(dim=1)
        assert float((rows - 1).abs().max()) < 2e-5
    # single-particle energies <psi|h|psi> from complex64 states: rounding of
    # the 2.2e5-term contractions, amplified by the kinetic/potential
    # cancellation, leaves a few keV at this stage (the CUDA-core FP32 Gram
    # shows the same); the FP64 tail of the mixed driver removes it
    e32 = l32.sp_energy.cpu().numpy()
    e64 = l64.sp_energy.cpu().numpy()
    assert np.max(np.abs(np.sort(e32) - np.sort(e64))) < 2e-2


@pytest.mark.gpu
def test_rotation_tma_feed_matches_register_producers(monkeypatch):
    """One single-precision diagstep on Pb208 states (rotation tasks over
    48^3 x 2 grid points, three 72-output chunks for the neutrons) with the
    TMA-fed rotation (the default) and with its register-loaded producers
    (HFB_TMA_FEED=0 at context creation): the same three-term products, so
    the rotated states and the single-particle energies agree to
    single-precision rounding."""
    from hfb import config, static

    def run():
        st = config.setup(config.case_dict("Pb208"), dtype=torch.complex128)
        S = {k: st[k] for k in static._STATE_KEYS}
        static.prepare(**S)
        for i in (1, 2):
            static.iterate(i, **S)
        static.to_precision(st, torch.complex64)
        static.diagstep(st["energies"], st["forces"], st["grids"], st["levels"], st["static"], True, True)
        torch.cuda.synchronize()
        st["grids"].ctx.check("diagstep")
        return st["levels"].psi.detach().clone(), st["levels"].sp_energy.detach().cpu().numpy().copy()

    p1, e1 = run()
    monkeypatch.setenv("HFB_TMA_FEED", "0")
    p2, e2 = run()
    assert float((p1 - p2).abs().max()) <= 1e-4 * float(p2.abs().max())
    assert np.max(np.abs(e1 - e2)) < 1e-3


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64], ids=["f64", "f32"])
def test_diagstep_overlapped_matches_sequential(monkeypatch, dtype):
    """The diagonalisation step with the H, G Gram launch, Newton-Schulz and
    the rotation's transposes overlapping the lambda eigensolve on side
    streams (the default) against the same step with one Gram launch and
    everything after it on the main stream (HFB_GRAM_SPLIT=0 at context
    creation), on Pb208 after two iterations: the FP64 Gram's tiles do not
    depend on the matrices computed with it, so FP64 agrees bit for bit.
    In single precision the tensor-core Gram's K slices are shared out by
    the number of matrices in the launch, so lambda differs at rounding
    level and the eigensolver picks another basis inside the degenerate
    (Kramers) pairs: the checks are gauge invariant -- each state of one
    run lies in the span of the other's (row norms of the overlap matrix
    per isospin) and the sorted single-particle energies agree."""
    from hfb import config, static

    def run():
        st = config.setup(config.case_dict("Pb208"), dtype=torch.complex128)
        S = {k: st[k] for k in static._STATE_KEYS}
        static.prepare(**S)
        for i in (1, 2):
            static.iterate(i, **S)
        if dtype != torch.complex128:
            static.to_precision(st, dtype)
        static.diagstep(st["energies"], st["forces"], st["grids"], st["levels"], st["static"], True, True)
        torch.cuda.synchronize()
        st["grids"].ctx.check("diagstep")
        lv = st["levels"]
        run.geo = (st["grids"].wxyz, lv.npsi[0], lv.nstmax)
        return (lv.psi.detach().clone(), lv.lagrange.detach().clone(), lv.sp_energy.detach().cpu().numpy().copy(),
                st["static"].hmatrix.detach().cpu().numpy().copy())

    p1, l1, e1, h1 = run()
    monkeypatch.setenv("HFB_GRAM_SPLIT", "0")
    p2, l2, e2, h2 = run()
    if dtype == torch.complex128:
        assert torch.equal(p1, p2) and torch.equal(l1, l2)
        assert np.array_equal(e1, e2) and np.array_equal(h1, h2)
    else:
        wxyz, n0, ns = run.geo
        for sl in (slice(0, n0), slice(n0, ns)):
            a = p1[sl].reshape(sl.stop - sl.start, -1).to(torch.complex128)
            b = p2[sl].reshape(sl.stop - sl.start, -1).to(torch.complex128)
            rows = (((a.conj() @ b.T) * wxyz).abs() ** 2).sum(dim=1)
            assert float((rows - 1).abs().max()) < 2e-5
        # <psi|h|psi> from complex64 states carries a few keV of rounding at
        # this stage (measured 6.4e-3 MeV between the two forms), the bound
        # of the single- against double-precision test above
        assert np.max(np.abs(np.sort(e1) - np.sort(e2))) < 2e-2


def _near_diag_hermitian(n, seed, scale, kramers=True):
    """Hermitian test matrix close to diagonal: spread diagonal with exactly
    degenerate pairs (as time reversal gives), plus a random Hermitian
    coupling of size ``scale``."""
    rng = np.random.default_rng(seed)
    d = np.sort(rng.uniform(-60.0, 40.0, (n + 1) // 2))
    diag = np.repeat(d, 2)[:n] if kramers else np.sort(rng.uniform(-60.0, 40.0, n))
    h = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    h = scale * (h + h.conj().T) / 2
    return np.diag(diag) + h


@pytest.mark.gpu
@pytest.mark.parametrize("n,scale,kramers", [(140, 1e-3, True), (96, 1e-2, True), (40, 1e-4, False),
                                             (140, 5.0, True)])
def test_eigh_near_diagonal(n, scale, kramers):
    """hfb_eigh_near_diagonal (iterative refinement + exact cluster solves,
    Jacobi when it does not apply; the last case is far from diagonal)
    against numpy: eigenvalues, residual ||A V - V W|| and orthonormality."""
    import hfb
    from hfb._lib import call, ptr, stream_ptr
    p = hfb.params.init_params()
    g = hfb.grids.init_grids(p, nx=8, ny=8, nz=8, dx=1.0, dy=1.0, dz=1.0)
    nb = 3
    a = np.stack([_near_diag_hermitian(n, 5 + k, scale, kramers) for k in range(nb)])
    # the solver reads the lower triangle only
    a_in = np.tril(a) + np.triu(np.full_like(a, 7.0 + 3.0j), 1)
    ta = T(a_in)
    w = torch.zeros((nb, n), dtype=torch.float64, device="cuda")
    v = torch.zeros((nb, n, n), dtype=torch.complex128, device="cuda")
    call("hfb_eigh_near_diagonal", g.ctx.handle, nb, n, n, ptr(ta), ptr(w), ptr(v), stream_ptr())
    torch.cuda.synchronize()
    wv, vv = w.cpu().numpy(), v.cpu().numpy()
    for k in range(nb):
        ref = np.linalg.eigvalsh(a[k])
        amax = np.abs(ref).max()
        assert np.max(np.abs(wv[k] - ref)) < 1e-12 * amax * n
        assert np.max(np.abs(a[k] @ vv[k] - vv[k] * wv[k][None, :])) < 1e-11 * amax
        assert np.max(np.abs(vv[k].conj().T @ vv[k] - np.eye(n))) < 1e-12


@pytest.mark.gpu
def test_single_precision_iterations_tensor_cores_match_cuda_cores(monkeypatch):
    """Five single-precision iterations of O16 (24^3) with the tensor-core
    kernels (hpsi, Gram, rotation) and with HFB_NO_TCGEN05=1 at context
    creation (FFT hpsi and CUDA-core contractions) agree to single-precision
    accuracy."""
    from hfb import config, static

    def run():
        st = config.setup(config.case_dict("O16"), dtype=torch.complex64)
        S = {k: st[k] for k in static._STATE_KEYS}
        static.prepare(**S)
        for i in range(1, 6):
            static.iterate(i, **S)
        return st["energies"].ehf, st["levels"].sp_energy.detach().cpu().numpy().copy()

    e1, s1 = run()
    monkeypatch.setenv("HFB_NO_TCGEN05", "1")
    e2, s2 = run()
    assert abs(e1 - e2) < 5e-3, (e1, e2)
    assert np.max(np.abs(s1 - s2)) < 2e-2


@pytest.mark.parametrize("name", ["o16_n16", "ne20_vdi_n16", "o18_dddi_n16", "triaxial_n16"])
def test_observables_against_reference(name):
    """hfb_observables (device FP64 reductions + 3x3 Jacobi) against the
    reference's calculate_complete_observables on the golden densities,
    through the Python mirror; with summed currents for the triaxial case."""
    import types
    import hfb
    z = np.load(os.path.join(GOLDEN, "observables_n16.npz"))
    n, dx, dy, dz = z[f"{name}_grid"]
    p = hfb.params.init_params()
    g = hfb.grids.init_grids(p, nx=int(n), ny=int(n), nz=int(n), dx=dx, dy=dy, dz=dz)
    nn, nz = z[f"{name}_nucleons"]
    rho = T(z[f"{name}_rho"])
    cur = T(z[f"{name}_current"]) if f"{name}_current" in z.files else None
    lv = types.SimpleNamespace(nneut=int(nn), nprot=int(nz))
    o = hfb.output.calculate_complete_observables(types.SimpleNamespace(rho=rho), lv, g, p, cur)
    g.ctx.check("observables")
    ref = lambda k: z[f"{name}_{k}"]
    for k in ("pnr", "pnrtot", "cm", "cmtot", "dipole_isovector", "rms", "rmstot", "x2m", "x2mtot", "pcm"):
        np.testing.assert_allclose(np.asarray(getattr(o, k)), ref(k), rtol=1e-11, atol=1e-12, err_msg=k)
    qs = max(1.0, float(np.max(np.abs(ref("q20")))))
    for k in ("q20", "q22", "q20tot", "q22tot"):
        np.testing.assert_allclose(np.asarray(getattr(o, k)), ref(k), rtol=0, atol=1e-10 * qs, err_msg=k)
    for k in ("q20T1", "beta20tot", "beta22tot", "beta"):
        np.testing.assert_allclose(getattr(o, k), ref(k), rtol=0, atol=1e-11, err_msg=k)
    if ref("beta") > 0.01:
        assert abs(o.gamma - ref("gamma")) < 1e-8
    assert np.allclose(o.qmat, np.transpose(o.qmat, (1, 0, 2)))
