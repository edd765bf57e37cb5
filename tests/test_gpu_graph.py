"""Iterations replayed as CUDA graphs (hfb.graph) against the ordinary
driver.  The captured work is the same sequence of library launches and
the device step-size rule is the host's rule in the same double precision,
so the energy histories agree to rounding (1e-9 MeV here), one instance
alone and two different instances in one graph."""
import copy

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _case(n=16, scale=1.0):
    from hfb import config
    from hfb.adjoint import force_overrides, theta_of
    from hfb.forces import init_forces
    case = config.case_dict("O16", grid=dict(nx=n, ny=n, nz=n), static=dict(inibcs=6, inidiag=6))
    if scale != 1.0:
        t0 = theta_of(init_forces(None, name="SLy4"))["t0"]
        case = force_overrides(case, {"t0": t0 * scale})
    return case


def _plain(case, iters, dtype):
    from hfb import config, static
    st = config.setup(copy.deepcopy(case), dtype=dtype)
    S = {k: st[k] for k in static._STATE_KEYS}
    static.prepare(**S)
    E = []
    for i in range(1, iters + 1):
        static.iterate(i, **S)
        E.append(st["energies"].ehf)
    return np.array(E)


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
def test_graph_replay_matches_plain_iterations(dtype):
    from hfb import config, graph
    case = _case()
    ref = _plain(case, 52, dtype)
    r = graph.GraphRun(config.setup(copy.deepcopy(case), dtype=dtype))
    r.start()
    r.plain(r.steady_from())                 # 12 ordinary iterations
    bg = graph.BatchGraph([r], block=10).capture()
    for _ in range(4):
        bg.replay()
    bg.release()
    E = np.array(r.E)
    assert len(E) == 52
    tol = 1e-9 if dtype == torch.complex128 else 1e-6
    assert np.max(np.abs(E - ref)) < tol


def test_two_instances_in_one_graph_match_their_solo_runs():
    from hfb import config, graph
    cases = [_case(16), _case(24, scale=1.01)]
    refs = [_plain(c, 32, torch.complex128) for c in cases]
    runs = [graph.GraphRun(config.setup(copy.deepcopy(c), dtype=torch.complex128)) for c in cases]
    for r in runs:
        r.start()
        r.plain(r.steady_from())
    bg = graph.BatchGraph(runs, block=10).capture()
    for _ in range(2):
        bg.replay()
    bg.release()
    for r, ref in zip(runs, refs):
        assert np.max(np.abs(np.array(r.E) - ref)) < 1e-9
    # the second instance leaves; the batch is recomposed from the first
    # one's existing capture, which carries on where it stopped
    g0 = runs[0].graph
    runs[1].drop_graph()
    bg = graph.BatchGraph(runs[:1], block=10).capture()
    assert runs[0].graph is g0
    bg.replay()
    bg.release()
    ref = _plain(cases[0], 42, torch.complex128)
    assert np.max(np.abs(np.array(runs[0].E) - ref)) < 1e-9


def test_graph_solve_mixed_precision_converges_like_the_host_driver():
    from hfb import config, graph, static
    case = _case(24)
    st = config.setup(copy.deepcopy(case), dtype=torch.complex64)
    hist, _ = static.statichf_mixed(st, maxiter=3000, stop_mev=5e-6, fp32_min_points=0)
    res = graph.solve([config.setup(copy.deepcopy(case), dtype=torch.complex64)], stop_mev=5e-6, maxiter=3000,
                      fp32_min_points=0)
    assert res[0]["switch"] is not None and res[0]["switch"] > 0
    assert abs(res[0]["E"][-1] - hist[-1][1]) < 1e-3


def test_hpsi_tuner_times_every_kernel_and_caches_the_choice():
    from hfb import config, static, tune
    st = config.setup(_case(24), dtype=torch.complex64)
    static.prepare(**{k: st[k] for k in static._STATE_KEYS})
    best = tune.tune_hpsi(st)
    assert best in tune.KINDS.values()
    (entry,) = [v for k, v in tune.cache().items() if k.startswith("n24_")]
    assert set(entry["seconds"]) == set(tune.KINDS.values()) and min(entry["seconds"].values()) > 0
    assert entry["best"] == min(entry["seconds"], key=entry["seconds"].get)
    assert tune.tune_hpsi(st) == best      # from the cache
