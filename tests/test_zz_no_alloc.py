"""The allocation-free Coulomb solve (hfb_poisson_noalloc) against the
allocating one (hfb_poisson), called through the C ABI.

Kept in its own file, collected last, so a run that stops at the first
failure has run every other test first; it also passes alone in a fresh
process (the first call on the device performs the one-time address lookup).
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _solve(lib_name, g, rho):
    from hfb._lib import call, ptr, stream_ptr
    w = torch.full((g.nx, g.ny, g.nz), float("nan"), dtype=torch.float64, device="cuda")
    call(lib_name, g.ctx.handle, ptr(rho[1].contiguous()), ptr(w), stream_ptr())
    torch.cuda.synchronize()
    return w.cpu().numpy()


@pytest.mark.parametrize("n,d,periodic", [(16, 1.0, False), (32, 0.8, False), (32, 0.8, True), (48, 0.8, True)])
def test_poisson_noalloc_matches_allocating_solve_twice(n, d, periodic):
    """Non-periodic grids (doubled Coulomb grid 2n, pruned padding) and
    periodic ones (Coulomb grid n, 1/k^2 Green's function): the periodic
    48^3 grid fills 48^3 of the 64^3 buffer."""
    import hfb
    g = hfb.grids.init_grids(hfb.params.init_params(), nx=n, ny=n, nz=n, dx=d, dy=d, dz=d, periodic=periodic)
    x = (torch.arange(n, dtype=torch.float64, device="cuda") - (n - 1) / 2) * d
    r2 = x[:, None, None] ** 2 + x[None, :, None] ** 2 + (1.2 * x[None, None, :]) ** 2
    for call_no in range(2):           # two calls in a row share the one buffer
        rho = torch.stack([0.08 * torch.exp(-r2 / 9.0), (0.07 + 0.01 * call_no) * torch.exp(-r2 / 8.0)]).contiguous()
        ref = _solve("hfb_poisson", g, rho)
        got = _solve("hfb_poisson_noalloc", g, rho)
        assert np.all(np.isfinite(got))
        assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_poisson_noalloc_rejects_large_grid():
    import hfb
    from hfb._lib import load, ptr, stream_ptr, HFB_OK
    g = hfb.grids.init_grids(hfb.params.init_params(), nx=48, ny=48, nz=48, dx=0.8, dy=0.8, dz=0.8)
    rho = torch.zeros((2, 48, 48, 48), dtype=torch.float64, device="cuda")
    w = torch.zeros((48, 48, 48), dtype=torch.float64, device="cuda")
    r = load().hfb_poisson_noalloc(g.ctx.handle, ptr(rho[1]), ptr(w), stream_ptr())
    assert r == 2   # HFB_ERR_UNSUPPORTED_GRID: the doubled 96^3 grid exceeds the fixed 64^3 buffer
    torch.cuda.synchronize()
    assert int(torch.count_nonzero(w)) == 0   # rejected before anything ran
