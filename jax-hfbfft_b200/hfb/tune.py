"""Kernel choice by measurement: the single-precision hpsi kernel of a grid
context (bf16 three-term or tf32 three-term tensor-core kernels, or the FFT
kernels on CUDA cores) timed on the instance's own states and potentials,
the fastest kept for the context and cached per (grid points, spacings,
states, neutron states).

    from hfb import tune
    kind = tune.tune_hpsi(state)          # state from hfb.config.setup, complex64

The cache lives for the process; ``HFB_TUNE_CACHE=<file>`` also keeps it in
a JSON file between processes.
"""
import json
import os

import torch

from ._lib import call, ptr, stream_ptr, prec_of

KINDS = {0: "bf16x3", 1: "tf32x3", 2: "fft"}
_cache = {}


def _key(grids, ns, nn):
    return f"n{grids.nx}_d{grids.dx:.4f}_{grids.dy:.4f}_{grids.dz:.4f}_s{ns}_nn{nn}"


def _load():
    p = os.environ.get("HFB_TUNE_CACHE")
    if p and os.path.exists(p):
        with open(p) as f:
            _cache.update(json.load(f))


def _save():
    p = os.environ.get("HFB_TUNE_CACHE")
    if p:
        with open(p, "w") as f:
            json.dump(_cache, f, indent=1, sort_keys=True)


def time_hpsi(state, kind, reps=5, warm=2):
    """Mean seconds of one hpsi over all states with kernel ``kind``."""
    g, lv, mf = state["grids"], state["levels"], state["meanfield"]
    call("hfb_set_hpsi_kernel", g.ctx.handle, int(kind))
    psi = lv.psi
    mf.pack(psi.dtype)
    out = torch.empty_like(psi)
    ns, nn = lv.nstmax, lv.npsi[0]
    wt = torch.ones(ns, dtype=torch.float64, device="cuda")
    wu = torch.zeros(ns, dtype=torch.float64, device="cuda")

    def once():
        call("hfb_hpsi", g.ctx.handle, prec_of(psi), ptr(mf.pot), ns, nn, ptr(psi), ptr(wt), ptr(wu), ptr(out),
             None, None, stream_ptr())

    for _ in range(warm):
        once()
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(reps):
        once()
    e1.record(s)
    torch.cuda.synchronize()
    g.ctx.check("hpsi tuning")
    return e0.elapsed_time(e1) / 1e3 / reps


def tune_hpsi(state, kinds=(0, 1, 2), reps=5):
    """Pick the fastest single-precision hpsi kernel for this instance's
    grid and state count (cached), set it on the context and return its
    name.  FP64 states always use the FFT kernels; nothing is tuned."""
    g, lv = state["grids"], state["levels"]
    if lv.psi.dtype != torch.complex64:
        return "fft"
    if not _cache:
        _load()
    key = _key(g, lv.nstmax, lv.npsi[0])
    if key not in _cache:
        times = {KINDS[k]: time_hpsi(state, k, reps=reps) for k in kinds}
        best = min(times, key=times.get)
        _cache[key] = dict(best=best, seconds=times)
        _save()
    best = _cache[key]["best"]
    call("hfb_set_hpsi_kernel", g.ctx.handle, {v: k for k, v in KINDS.items()}[best])
    return best


def cache():
    return dict(_cache)
