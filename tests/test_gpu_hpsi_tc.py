"""The two single-precision tensor-core hpsi kernels against the FP64 oracle.

``hpsi_bf3_kernel`` (the default; bf16 three-term operands, two CTAs per SM)
and ``hpsi_tc_kernel`` (tf32 three-term, selected with HFB_HPSI_KERNEL=tf32x3 when
the grid context is created) on every grid they serve, with unequal
spacings (one set of derivative matrices per axis), states of both
isospins spanning several scheduling groups, weights and all three outputs.
Both carry about 24 significant bits through the derivative GEMMs, so the
bound is 4e-6 relative (max |diff| / max |ref|) -- well inside the 1e-4
the FP32 path's other tests allow.
"""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 4e-6


def rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _case(n, ns, seed):
    from oracle import model, meanfield as omf
    rng = np.random.default_rng(seed)
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
    psi = (rng.standard_normal((ns, 2, n, n, n)) + 1j * rng.standard_normal((ns, 2, n, n, n))) * w
    return d, g, mfo, psi, rng.uniform(0.2, 1.0, ns), rng.uniform(0.0, 0.5, ns)


def _run(n, d, mfo, psi, wt, wu, nn, tf32):
    import hfb
    from hfb._lib import call, ptr, stream_ptr, prec_of
    old = os.environ.get("HFB_HPSI_KERNEL")
    os.environ["HFB_HPSI_KERNEL"] = "tf32x3" if tf32 else "bf16x3"
    try:
        gg = hfb.grids.init_grids(hfb.params.init_params(), nx=n, ny=n, nz=n, dx=d[0], dy=d[1], dz=d[2])
    finally:
        if old is None:
            del os.environ["HFB_HPSI_KERNEL"]
        else:
            os.environ["HFB_HPSI_KERNEL"] = old
    dtype = torch.complex64
    mf = hfb.meanfield.init_meanfield(gg, dtype)
    for k in ("upot", "bmass", "v_pair", "aq", "spot", "wlspot"):
        getattr(mf, k).copy_(torch.from_numpy(np.ascontiguousarray(getattr(mfo, k))).cuda())
    mf.pack(dtype)
    pt = torch.from_numpy(psi).cuda().to(dtype).contiguous()
    outs = [torch.empty_like(pt) for _ in range(3)]
    wt_t = torch.from_numpy(wt).cuda()
    wu_t = torch.from_numpy(wu).cuda()
    ns = psi.shape[0]
    n0 = hfb._lib.launch_count()
    call("hfb_hpsi", gg.ctx.handle, prec_of(pt), ptr(mf.pot), ns, nn, ptr(pt), ptr(wt_t), ptr(wu_t),
         ptr(outs[0]), ptr(outs[1]), ptr(outs[2]), stream_ptr())
    gg.ctx.check("hpsi")
    return outs, hfb._lib.launch_count() - n0


@pytest.mark.parametrize("n,ns", [(24, 37), (32, 9), (40, 6), (48, 11)])
@pytest.mark.parametrize("tf32", [False, True], ids=["bf16x3", "tf32x3"])
def test_tensor_core_hpsi_against_oracle(n, ns, tf32):
    from oracle import meanfield as omf
    d, g, mfo, psi, wt, wu = _case(n, ns, 100 + n)
    nn = ns // 2 + 1
    outs, launches = _run(n, d, mfo, psi, wt, wu, nn, tf32)
    assert launches >= 2   # field repack + the tensor-core kernel ran
    for iq, sl in ((0, slice(0, nn)), (1, slice(nn, ns))):
        r = omf.hpsi01(g, mfo, iq, wt[sl], wu[sl], psi[sl])
        for o, ref, tag in zip(outs, r, ("pout", "pout_mf", "pout_del")):
            e = rel(o[sl], ref)
            assert e < TOL, (iq, tag, e)
