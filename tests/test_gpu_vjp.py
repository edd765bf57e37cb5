"""Reverse-mode derivatives of hpsi and of the densities (hfb.vjp) on the
device: against the oracle's VJPs (oracle/vjp.py, itself checked against
central differences on the CPU), and through torch.autograd against central
differences of the device forward maps.  FP64 states at 16^3 with
anisotropic spacings, 5 states (3 neutrons, 2 protons), per-state
occupation and pairing weights and random fields: hpsi is linear and the
densities quadratic, so the bars are 1e-10 relative; the composite
nonlinear loss is held to 1e-6 (central-difference truncation)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

N, D, NS, NN = 16, (0.9, 1.0, 1.1), 5, 3
FIELDS = ("upot", "bmass", "v_pair", "aq", "spot", "wlspot")
DENS = ("rho", "chi", "tau", "current", "sdens", "sodens")


@pytest.fixture(scope="module")
def setup():
    import hfb
    from oracle import model
    rng = np.random.default_rng(11)
    gg = hfb.grids.init_grids(hfb.params.init_params(), nx=N, ny=N, nz=N, dx=D[0], dy=D[1], dz=D[2])
    go = model.init_grids(N, N, N, *D)
    x = [(np.arange(N) - (N - 1) / 2) * d for d in D]
    r2 = x[0][:, None, None] ** 2 + x[1][None, :, None] ** 2 + x[2][None, None, :] ** 2
    env = np.exp(-r2 / 12.0)
    rc = lambda *s: (rng.standard_normal(s) + 1j * rng.standard_normal(s)) * env
    f = {k: rng.standard_normal((2, N, N, N)) for k in ("upot", "bmass", "v_pair")}
    f.update({k: rng.standard_normal((2, 3, N, N, N)) for k in ("aq", "spot", "wlspot")})
    return dict(rng=rng, gg=gg, go=go, psi=rc(NS, 2, N, N, N), yb=rc(NS, 2, N, N, N), v=rc(NS, 2, N, N, N),
                w=rng.uniform(0.2, 1.0, NS), wu=rng.uniform(0.0, 0.5, NS), f=f)


def _t(a, dtype=None):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda() if dtype is None else torch.from_numpy(a).cuda().to(dtype)


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def test_hpsi_vjp_matches_oracle(setup):
    from hfb import vjp
    from oracle import meanfield as omf, vjp as ovjp
    s = setup
    gg, go = s["gg"], s["go"]
    fields = {k: _t(v) for k, v in s["f"].items()}
    psi, yb = _t(s["psi"]), _t(s["yb"])
    w, wu = _t(s["w"]), _t(s["wu"])
    pot = vjp._pack(gg, fields, torch.complex128).pot
    pb, bars = vjp.hpsi_vjp(gg, pot, psi, NN, w, wu, yb)
    mfo = omf.init_meanfield(go)
    for k, v in s["f"].items():
        setattr(mfo, k, v)
    for iq, sl in ((0, slice(0, NN)), (1, slice(NN, NS))):
        pbo, barso = ovjp.hpsi_vjp(go, mfo, iq, s["w"][sl], s["wu"][sl], s["psi"][sl], s["yb"][sl])
        assert _rel(pb[sl].cpu().numpy(), pbo) <= 1e-10
        for k in FIELDS:
            assert _rel(bars[k][iq].cpu().numpy(), barso[k]) <= 1e-10, k


def test_densities_vjp_matches_oracle(setup):
    from hfb import vjp
    from oracle import vjp as ovjp
    s = setup
    rng = np.random.default_rng(5)
    fb = {k: rng.standard_normal((2, N, N, N) if k in ("rho", "chi", "tau") else (2, 3, N, N, N)) for k in DENS}
    pb = vjp.densities_vjp(s["gg"], _t(s["psi"]), NN, _t(s["w"]), _t(s["wu"]), {k: _t(v) for k, v in fb.items()})
    for iq, sl in ((0, slice(0, NN)), (1, slice(NN, NS))):
        pbo = ovjp.densities_vjp(s["go"], s["w"][sl], s["wu"][sl], s["psi"][sl], iq, {k: v[iq] for k, v in fb.items()})
        assert _rel(pb[sl].cpu().numpy(), pbo) <= 1e-10


def _dot(a, b):
    return float(torch.sum((torch.conj(a) * b).real))


def test_hpsi_autograd_matches_central_differences(setup):
    from hfb import vjp
    s = setup
    gg = s["gg"]
    psi = _t(s["psi"]).requires_grad_(True)
    fields = {k: _t(v).requires_grad_(True) for k, v in s["f"].items()}
    yb, v = _t(s["yb"]), _t(s["v"])
    w, wu = _t(s["w"]), _t(s["wu"])

    def L(p, f):
        return _dot(yb, vjp.hpsi(p, f, gg, NN, w, wu))

    out = vjp.hpsi(psi, fields, gg, NN, w, wu)
    torch.sum((torch.conj(yb) * out).real).backward()
    e = 1e-3
    with torch.no_grad():
        fd = (L(psi + e * v, fields) - L(psi - e * v, fields)) / (2 * e)
        an = _dot(psi.grad, v)
        assert abs(an - fd) <= 1e-10 * abs(fd)
        for k in FIELDS:
            Q = torch.randn_like(fields[k])
            fp = {j: (x + e * Q if j == k else x) for j, x in fields.items()}
            fm = {j: (x - e * Q if j == k else x) for j, x in fields.items()}
            fd = (L(psi, fp) - L(psi, fm)) / (2 * e)
            an = float(torch.sum(fields[k].grad * Q))
            assert abs(an - fd) <= 1e-10 * max(abs(fd), 1.0), k


def test_densities_autograd_matches_central_differences(setup):
    from hfb import vjp
    s = setup
    gg = s["gg"]
    w, wu = _t(s["w"]), _t(s["wu"])
    psi = _t(s["psi"]).requires_grad_(True)
    v = _t(s["v"])
    gen = torch.Generator(device="cuda").manual_seed(3)
    d0 = vjp.densities(psi, gg, NN, w, wu)
    fb = {k: torch.randn(x.shape, dtype=torch.float64, device="cuda", generator=gen) for k, x in d0.items()}

    def L(p):
        d = vjp.densities(p, gg, NN, w, wu)
        return sum(torch.sum(fb[k] * d[k]) for k in DENS)

    L(psi).backward()
    e = 1e-3
    with torch.no_grad():
        fd = float(L(psi + e * v) - L(psi - e * v)) / (2 * e)
        assert abs(_dot(psi.grad, v) - fd) <= 1e-10 * abs(fd)


def test_composite_loss_through_densities_and_hpsi(setup):
    """L = sum_s Re<psi_s | h[U(rho), B(tau)] psi_s> + int rho^2, with
    U = -3 rho and B = 0.5 + 0.1 tau: psi enters the densities, the fields
    and hpsi; autograd's directional derivative against central
    differences (relative step 1e-5)."""
    from hfb import vjp
    s = setup
    gg = s["gg"]
    w, wu = _t(s["w"]), _t(s["wu"])
    psi = _t(s["psi"]).requires_grad_(True)
    v = _t(s["v"])
    zeros3 = torch.zeros((2, 3, N, N, N), dtype=torch.float64, device="cuda")
    zeros = torch.zeros((2, N, N, N), dtype=torch.float64, device="cuda")

    def L(p):
        d = vjp.densities(p, gg, NN, w, wu)
        f = dict(upot=-3.0 * d["rho"], bmass=0.5 + 0.1 * d["tau"], v_pair=zeros, aq=zeros3, spot=zeros3,
                 wlspot=zeros3)
        y = vjp.hpsi(p, f, gg, NN, 1.0, 0.0)
        return torch.sum((torch.conj(p) * y).real) + torch.sum(d["rho"] ** 2)

    L(psi).backward()
    e = 1e-5
    with torch.no_grad():
        fd = float(L(psi + e * v) - L(psi - e * v)) / (2 * e)
        an = _dot(psi.grad, v)
        assert abs(an - fd) <= 1e-6 * abs(fd), (an, fd)
