"""FP64 Gram contractions C_a = wxyz Psi^H X_a and the rotation
[psi U | psi L] on the FP64 tensor cores (HFB_F64_MMA=1, mma.sync m8n8k4
.f64) and on CUDA cores, against NumPy (complex128 GEMMs): 1e-12 relative
(max |diff| / max |ref|).  The rotation is exercised through
hfb_natural_end, whose states are psi cm and psi (cm htran)."""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _ctx(n, kind):
    import hfb
    old = os.environ.get("HFB_F64_MMA")
    os.environ["HFB_F64_MMA"] = "1" if kind == "dmma" else "0"
    try:
        return hfb.grids.init_grids(hfb.params.init_params(), nx=n, ny=n, nz=n, dx=0.8, dy=0.8, dz=0.8)
    finally:
        if old is None:
            del os.environ["HFB_F64_MMA"]
        else:
            os.environ["HFB_F64_MMA"] = old


@pytest.mark.parametrize("kind", ["dmma", "simt"])
@pytest.mark.parametrize("n,ns", [(16, 7), (24, 61), (32, 100)])
def test_gram_f64_against_numpy(kind, n, ns):
    from hfb._lib import call, ptr, stream_ptr, HFB_F64
    rng = np.random.default_rng(ns)
    K = 2 * n ** 3
    psi = rng.standard_normal((ns, K)) + 1j * rng.standard_normal((ns, K))
    ham = rng.standard_normal((ns, K)) + 1j * rng.standard_normal((ns, K))
    hmf = rng.standard_normal((ns, K)) + 1j * rng.standard_normal((ns, K))
    vp = rng.standard_normal(n ** 3)
    g = _ctx(n, kind)
    P, H, M = (torch.from_numpy(a).cuda() for a in (psi, ham, hmf))
    V = torch.from_numpy(vp).cuda()
    out = torch.zeros((4, ns, ns), dtype=torch.complex128, device="cuda")
    w = 0.512
    call("hfb_gram", g.ctx.handle, HFB_F64, 0, ns, 15, ptr(P), ptr(H), ptr(M), ptr(V), w, ptr(out), stream_ptr())
    g.ctx.check("gram")
    vpsi = psi * np.tile(vp, 2)[None, :]
    refs = [w * np.conj(psi) @ x.T for x in (psi, ham, hmf, vpsi)]
    o = out.cpu().numpy()
    iu = np.triu_indices(ns)
    for a, r in enumerate(refs):
        if a == 1:
            e = np.max(np.abs(o[a] - r)) / np.max(np.abs(r))
        else:
            # matrices 0, 2, 3 are Hermitian in the iteration (one set of
            # vectors; h psi, v_pair psi with h, v_pair Hermitian): computed
            # on the upper triangle and mirrored -- with the random hmfpsi
            # here only the upper triangle is defined
            e = np.max(np.abs(o[a][iu] - r[iu])) / np.max(np.abs(r[iu]))
            # off the diagonal the lower triangle is the exact mirror; the
            # diagonal keeps the rounding-level imaginary part of its sum
            off = ~np.eye(ns, dtype=bool)
            assert np.array_equal(o[a][off], np.conj(o[a].T)[off])
            if a != 2:            # random hmfpsi: its diagonal is not real
                assert np.max(np.abs(np.diag(o[a]).imag)) <= 1e-13 * np.max(np.abs(o[a]))
        assert e < 1e-12, (a, e)


@pytest.mark.parametrize("kind", ["dmma", "simt"])
def test_rotation_f64_through_natural(kind):
    """hfb_natural on the reference's seeded 8^3 inputs (whole blocks) with
    the rotation on each FP64 kernel, against the oracle's restatement."""
    import types
    import hfb
    from conftest import GOLDEN
    from oracle import static as ost
    d = dict(np.load(os.path.join(GOLDEN, "natural_n8.npz")))
    old = os.environ.get("HFB_F64_MMA")
    os.environ["HFB_F64_MMA"] = "1" if kind == "dmma" else "0"
    try:
        g = hfb.grids.init_grids(hfb.params.init_params(), nx=8, ny=8, nz=8, dx=0.9, dy=0.9, dz=0.9)
    finally:
        if old is None:
            del os.environ["HFB_F64_MMA"]
        else:
            os.environ["HFB_F64_MMA"] = old
    T = lambda k: torch.from_numpy(np.ascontiguousarray(d[f"e0_in_{k}"])).cuda()   # noqa: E731
    lv = types.SimpleNamespace(nneut=3, nprot=2, npsi=[4, 3], nstmax=7)
    lvo = types.SimpleNamespace(nneut=3, nprot=2, npsi=[4, 3], nstmax=7)
    for k in ("psi", "lagrange", "sp_energy", "wocc", "wguv", "pairwg", "wstates", "deltaf"):
        setattr(lv, k, T(k))
        setattr(lvo, k, d[f"e0_in_{k}"].copy())
    lv.psi_spare = torch.zeros_like(lv.psi)
    st = types.SimpleNamespace(e0bas=10.0, delstepbas=2.0)
    sto = types.SimpleNamespace(e0bas=10.0, delstepbas=2.0)
    for k in ("hmatrix", "gapmatrix", "symcond", "lambda_save"):
        setattr(st, k, T(k))
        setattr(sto, k, d[f"e0_in_{k}"].copy())
    for iq in range(2):
        hfb.static.hfb_natural(types.SimpleNamespace(ipair=0), g, lv, None, None, st, iq, 2)
        ost.hfb_natural(lvo, sto, iq, 2)
    for k in ("psi", "lagrange"):
        a = getattr(lv, k).cpu().numpy()
        b = getattr(lvo, k)
        assert np.max(np.abs(a - b)) < 1e-12 * np.max(np.abs(b)), k
