"""The measurement rules of bench.py, on synthetic energy histories (no GPU):
the time-to-converge point is the first iteration, among the allowed ones
(FP64 iterations for the mixed run), after which every later energy stays
within the tolerance of the reference energy."""
import importlib.util
import os

from conftest import ROOT


def _bench():
    spec = importlib.util.spec_from_file_location("bench_rules", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_converged_index_first_point_that_stays_within_tolerance():
    b = _bench()
    e_ref, tol = -100.0, 1e-3
    E = [-90.0, -99.0, -99.9995, -100.002, -99.9996, -99.9999, -100.0]
    # index 2 is within 1 keV but index 3 leaves it again: the run converges at 4
    assert b.converged_index(E, e_ref, tol, [True] * len(E)) == 4
    # only FP64 iterations count for the mixed run (here from index 5 on)
    assert b.converged_index(E, e_ref, tol, [False] * 5 + [True] * 2) == 5
    # never within tolerance at the end: no time-to-converge
    assert b.converged_index(E[:4], e_ref, tol, [True] * 4) is None
    # within tolerance but no allowed iteration in the final stretch
    assert b.converged_index(E, e_ref, tol, [True] * 4 + [False] * 3) is None


def test_remaining_change_is_exact_on_a_geometric_tail():
    """The stopping and precision-switch rules read the geometric estimate
    of E_limit - E[-1]: exact on E_k = E_inf + A q^k, None while the
    history is short or its tail is not geometric (growing or oscillating
    differences)."""
    from hfb import static
    e_inf, a, q = -1635.6815, 3.0, 0.97
    E = [e_inf + a * q ** k for k in range(200)]
    rem = static.remaining_change(E)
    assert abs(rem - (e_inf - E[-1])) < 1e-9
    assert static.remaining_change(E[:50]) is None
    assert static.remaining_change([e_inf + (-1) ** k * 0.1 * 0.9 ** k for k in range(60)]) is None
    assert static.remaining_change([e_inf - 0.01 * k for k in range(60)]) is None
    assert static.remaining_change([e_inf] * 60) == 0.0
