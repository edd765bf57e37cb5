"""Sensitivities (hfb.adjoint) against central finite differences (relative
step 1e-4) of the self-consistent solution, on the Ca48 sensitivity
workload (32^3, dx 0.8 fm, 40 + 30 states, SLy4 + volume delta pairing):
the binding energy's explicit gradient for the eleven Skyrme couplings
(t0-t3, x0-x3, t4, b4p, alpha) and
both pairing strengths, and the proton rms radius's gradient by the
implicit adjoint (linear-response solve at the fixed point).  Ca48 is
doubly magic: its BCS gap all but collapses, the occupations are within
about 1e-5 of 0 or 1, and the response holds them fixed (the occupation
response is of the order of their distance from 0 / 1)."""
import numpy as np
import pytest
import torch


@pytest.fixture(scope="module")
def ca48():
    from hfb import config, adjoint
    case = config.case_dict("Ca48")
    st, E = adjoint.converge(case, tol=1e-11)
    return case, st


@pytest.mark.gpu
def test_coupling_gradient_matches_central_fd(ca48):
    """dE_bind/dtheta from the explicit derivative of the functional at the
    fixed point agrees with central differences (relative step 1e-4) to
    1e-4 relative for the Skyrme couplings."""
    from hfb import adjoint
    case, st = ca48
    names = list(adjoint.SKYRME)
    g = adjoint.coupling_gradient(st)
    fd = adjoint.fd_gradient(case, names, rel_step=1e-4, base=st, tol=1e-11)
    for n in names:
        assert abs(g[n] - fd[n]) <= 1e-4 * abs(fd[n]), (n, g[n], fd[n])
    # W0 moves t4 and b4p in proportion: its gradient is the chain rule of the two
    f = st["forces"]
    assert abs(g["W0"] - (g["t4"] + f.b4p / f.t4 * g["b4p"])) <= 1e-12 * abs(g["W0"])


@pytest.mark.gpu
def test_pairing_strength_gradient_collapsed_pairing(ca48):
    """Ca48 is doubly magic: the BCS gap collapses, epair is below 1 keV and
    dE/dv0 = -epair/v0 is below 1e-5 MeV per MeV fm^3; the central
    differences agree within that noise level."""
    from hfb import adjoint
    case, st = ca48
    g = adjoint.coupling_gradient(st)
    fd = adjoint.fd_gradient(case, ["v0neut", "v0prot"], rel_step=1e-4, base=st, tol=1e-11)
    for n in ("v0neut", "v0prot"):
        assert abs(g[n]) < 1e-5 and abs(fd[n]) < 1e-5


@pytest.mark.gpu
def test_coupling_gradient_with_bcs_pairing_cr48():
    """Cr48 (32^3, 32 + 32 states, volume-delta pairing with the 60 MeV soft
    window, open shells; a weak BCS solution, epair about 1 keV per
    isospin): dE_bind/dtheta for the eleven Skyrme couplings from the explicit
    derivative against central differences (relative step 1e-4) to 1e-4
    relative (measured on B200: at most 5.3e-5).  The pairing strengths are
    left out: there the reference's BCS (soft cutoff, floored u v) is not
    variational and the explicit -epair/v0 misses the occupation response
    (measured -4.6e-6 against +1.5e-6 MeV per MeV fm^3)."""
    from hfb import config, adjoint
    case = config.case_dict("Cr48")
    st, _ = adjoint.converge(case, tol=1e-11, maxiter=3000)
    names = list(adjoint.SKYRME)
    g = adjoint.coupling_gradient(st)
    fd = adjoint.fd_gradient(case, names, rel_step=1e-4, base=st, tol=1e-11, maxiter=3000)
    for n in names:
        assert abs(g[n] - fd[n]) <= 1e-4 * abs(fd[n]), (n, g[n], fd[n])


@pytest.mark.gpu
def test_binding_energy_autograd_function(ca48):
    """torch.autograd.Function wrapper: forward returns the converged E_bind,
    backward the coupling gradient."""
    from hfb import adjoint
    case, st = ca48
    names = ["t0", "power"]
    th0 = adjoint.theta_of(st["forces"])
    theta = torch.tensor([th0[n] for n in names], dtype=torch.float64, requires_grad=True)
    e = adjoint.binding_energy(theta, case, names, tol=1e-11)
    e.backward()
    g = adjoint.coupling_gradient(st)
    assert abs(float(e.detach()) - st["energies"].ehf) < 1e-8
    np.testing.assert_allclose(theta.grad.numpy(), [g[n] for n in names], rtol=1e-6)


@pytest.fixture(scope="module")
def ca48_states():
    """Ca48 converged until the proton rms radius itself is stationary to
    1e-13 fm (an energy criterion leaves the states converged only to about
    the square root of its tolerance)."""
    from hfb import config, adjoint
    case = config.case_dict("Ca48")
    st, R = adjoint.converge_states(case, tol_r=1e-13)
    return case, st


@pytest.mark.gpu
def test_rms_gradient_implicit_adjoint_matches_central_fd(ca48_states):
    """dr_rms(p)/dtheta for the eleven Skyrme couplings: the adjoint solve
    (CG on the occupied-virtual orbital Hessian) against central
    differences of the reconverged radius, 1e-4 relative (measured on B200:
    at most 8.4e-6, CG residual 7e-11 after 79 iterations)."""
    from hfb import adjoint
    case, st = ca48_states
    names = list(adjoint.SKYRME)
    g, info = adjoint.rms_gradient(st, names, tol=1e-9, allow_fractional=True)
    assert info["residual"] < 1e-9 and info["cg_iterations"] < 500
    fd = adjoint.fd_rms_gradient(case, names, rel_step=1e-4, base=st, tol_r=1e-13)
    for n in names:
        assert abs(g[n] - fd[n]) <= 1e-4 * abs(fd[n]), (n, g[n], fd[n])


@pytest.mark.gpu
def test_rms_gradient_pairing_strengths_vanish_with_collapsed_pairing(ca48_states):
    from hfb import adjoint
    case, st = ca48_states
    g, _ = adjoint.rms_gradient(st, ["v0neut", "v0prot"], tol=1e-8, allow_fractional=True)
    fd = adjoint.fd_rms_gradient(case, ["v0neut"], rel_step=1e-4, base=st, tol_r=1e-13)
    assert abs(g["v0neut"]) < 1e-9 and abs(g["v0prot"]) < 1e-9 and abs(fd["v0neut"]) < 1e-7
