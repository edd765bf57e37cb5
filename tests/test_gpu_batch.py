"""Concurrent parameter sweep (hfb.batch): instances solved side by side on
separate streams give the results they give alone."""
import pytest


def test_sweep_cases_are_seeded():
    from hfb import batch
    a = batch.sweep_cases(12, seed=5)
    b = batch.sweep_cases(12, seed=5)
    assert [x[0] for x in a] == [x[0] for x in b]
    assert all(abs(x[2]["t0"] - 1.0) <= 0.02 for x in a)
    assert a[0][1]["force"]["overrides"] == b[0][1]["force"]["overrides"]


@pytest.mark.gpu
def test_concurrent_sweep_matches_sequential():
    from hfb import batch
    cases = batch.sweep_cases(5, seed=11, species=["O16", "Ca40"])
    seq = batch.run_sweep(cases, workers=1, maxiter=400)
    con = batch.run_sweep(cases, workers=3, maxiter=400)
    for a, b in zip(seq, con):
        assert a["species"] == b["species"]
        assert a["ehf"] == b["ehf"] and a["iterations"] == b["iterations"]
    assert len({round(r["ehf"], 3) for r in seq}) > 1     # the couplings differ
