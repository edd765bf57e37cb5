"""Failure detection on the device, made to happen without faulting the GPU.

* A bounded wait that runs out: the timeout probe makes the first CTA of the
  next single-precision tensor-core hpsi launch wait on a device word that
  nothing writes, with a short wait limit.  The launch must end, latch
  HFB_ERR_TIMEOUT (read by the host), release its tensor memory, and leave
  the context usable: the same call afterwards gives the right result.
* A non-finite energy: a NaN planted on the host in a density makes the
  energy kernel latch HFB_ERR_NONFINITE, which the driver's per-iteration
  status check turns into an exception.
"""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _hpsi_inputs(n=24, ns=6, seed=3):
    import hfb
    from oracle import model, meanfield as omf
    rng = np.random.default_rng(seed)
    g = model.init_grids(n, n, n, 0.8, 0.8, 0.8)
    x = (np.arange(n) - (n - 1) / 2) * 0.8
    r2 = x[:, None, None] ** 2 + x[None, :, None] ** 2 + x[None, None, :] ** 2
    w = np.exp(-r2 / 20.0)
    mfo = omf.init_meanfield(g)
    mfo.upot = np.stack([-50 * w, -45 * w])
    mfo.bmass = np.stack([20 + 2 * w, 21 + 1.5 * w])
    mfo.v_pair = np.stack([-3 * w, -2 * w])
    psi = (rng.standard_normal((ns, 2, n, n, n)) + 1j * rng.standard_normal((ns, 2, n, n, n))) * w
    old = os.environ.get("HFB_HPSI_KERNEL")
    os.environ["HFB_HPSI_KERNEL"] = "bf16x3"   # the kernel with the timeout probe
    try:
        gg = hfb.grids.init_grids(hfb.params.init_params(), nx=n, ny=n, nz=n, dx=0.8, dy=0.8, dz=0.8)
    finally:
        if old is None:
            del os.environ["HFB_HPSI_KERNEL"]
        else:
            os.environ["HFB_HPSI_KERNEL"] = old
    mf = hfb.meanfield.init_meanfield(gg, torch.complex64)
    for k in ("upot", "bmass", "v_pair"):
        getattr(mf, k).copy_(torch.from_numpy(getattr(mfo, k)).cuda())
    mf.pack(torch.complex64)
    return gg, g, mfo, mf, psi


def _hpsi(gg, mf, psi_t, ns, nn):
    from hfb._lib import call, ptr, stream_ptr, prec_of
    out = torch.full_like(psi_t, float("nan"))
    call("hfb_hpsi", gg.ctx.handle, prec_of(psi_t), ptr(mf.pot), ns, nn, ptr(psi_t), None, None, ptr(out), None,
         None, stream_ptr())
    return out


def test_wait_timeout_is_reported_and_context_stays_usable():
    from hfb._lib import call, load, HFB_ERR_TIMEOUT
    from oracle import meanfield as omf
    gg, g, mfo, mf, psi = _hpsi_inputs()
    ns, nn = psi.shape[0], 3
    psi_t = torch.from_numpy(psi).cuda().to(torch.complex64).contiguous()
    assert gg.ctx.device_status() == 0
    call("hfb_set_wait_limit", gg.ctx.handle, 1000000)        # ~0.5 ms
    call("hfb_arm_timeout_probe", gg.ctx.handle)
    _hpsi(gg, mf, psi_t, ns, nn)
    torch.cuda.synchronize()                                   # the launch ended by itself
    assert gg.ctx.device_status() == HFB_ERR_TIMEOUT
    assert gg.ctx.device_status() == 0                         # reading the status clears it
    # the probe is spent and the tensor memory was released: a second
    # launch runs to completion and is right
    call("hfb_set_wait_limit", gg.ctx.handle, 2000000000)
    out = _hpsi(gg, mf, psi_t, ns, nn)
    assert gg.ctx.device_status() == 0
    for iq, sl in ((0, slice(0, nn)), (1, slice(nn, ns))):
        ref = omf.hpsi01(g, mfo, iq, 1.0, 0.0, psi[sl])[0]
        o = out[sl].cpu().numpy()
        assert np.max(np.abs(o - ref)) <= 1e-5 * np.max(np.abs(ref))
    assert load().hfb_set_wait_limit(gg.ctx.handle, 0) == 1   # HFB_ERR_ARG


def test_nonfinite_energy_is_latched_and_raised():
    import hfb
    from hfb import config, static
    from hfb._lib import HfbError, HFB_ERR_NONFINITE
    case = config.case_dict("O16", grid=dict(nx=16, ny=16, nz=16))
    st = config.setup(case)
    S = {k: st[k] for k in static._STATE_KEYS}
    static.prepare(**S)
    static.iterate(1, **S)                                     # a clean iteration first
    st["densities"].rho[0, 8, 8, 8] = float("nan")             # planted on the host side of the API
    hfb.energies.integ_energy(st["coulomb"], st["densities"], st["energies"], st["forces"], st["grids"],
                              st["levels"], st["params"], st["pairs"])
    assert st["grids"].ctx.device_status() == HFB_ERR_NONFINITE
    st["densities"].rho[0, 8, 8, 8] = float("nan")
    with pytest.raises(HfbError) as e:
        static.iterate(2, **S)
    assert e.value.code == HFB_ERR_NONFINITE
