"""Energy sensitivities (hfb.adjoint) against central finite differences of
the self-consistent binding energy, on the Ca48 sensitivity workload
(32^3, dx 0.8 fm, 40 + 30 states, SLy4 + volume delta pairing)."""
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
    names = ["t0", "x1", "t3", "power", "W0"]
    g = adjoint.coupling_gradient(st)
    fd = adjoint.fd_gradient(case, names, rel_step=1e-4, base=st, tol=1e-11)
    for n in names:
        assert abs(g[n] - fd[n]) <= 1e-4 * abs(fd[n]), (n, g[n], fd[n])


@pytest.mark.gpu
def test_pairing_strength_gradient_collapsed_pairing(ca48):
    """Ca48 is doubly magic: the BCS gap collapses, epair is below 1 keV and
    dE/dv0 = -epair/v0 is below 1e-5 MeV per MeV fm^3; the central
    differences agree within that noise level."""
    from hfb import adjoint
    case, st = ca48
    g = adjoint.coupling_gradient(st)
    fd = adjoint.fd_gradient(case, ["v0neut"], rel_step=1e-4, base=st, tol=1e-11)
    assert abs(g["v0neut"]) < 1e-5 and abs(fd["v0neut"]) < 1e-5


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
