"""FP64 Gram contractions C_a = wxyz Psi^H X_a on the FP64 tensor cores
(HFB_GRAM_F64=dmma, mma.sync m8n8k4 .f64) and on CUDA cores, against NumPy
(complex128 GEMM): 1e-12 relative (max |diff| / max |ref|)."""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _ctx(n, kind):
    import hfb
    old = os.environ.get("HFB_GRAM_F64")
    os.environ["HFB_GRAM_F64"] = kind
    try:
        return hfb.grids.init_grids(hfb.params.init_params(), nx=n, ny=n, nz=n, dx=0.8, dy=0.8, dz=0.8)
    finally:
        if old is None:
            del os.environ["HFB_GRAM_F64"]
        else:
            os.environ["HFB_GRAM_F64"] = old


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
    for a, r in enumerate(refs):
        e = np.max(np.abs(o[a] - r)) / np.max(np.abs(r))
        assert e < 1e-12, (a, e)
