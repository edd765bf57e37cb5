"""Parameter sweeps over many nuclei: independent self-consistent solves run
concurrently on one GPU.

Each instance (a nucleus and a set of Skyrme couplings) has its own grid
context and state buffers and runs the mixed-precision driver
(``static.statichf_mixed``: single-precision bulk, double-precision
refinement) on a CUDA stream of its own; a pool of host threads keeps
``workers`` instances in flight, so the small per-instance kernels of
different nuclei overlap on the GPU.  Instances share nothing on the
device, so each result is the one the instance gives alone.

``run_sweep_graph`` instead advances a group of instances together: after
their start-up iterations, blocks of iterations of every instance in the
group are captured into one CUDA graph (hfb.graph) and each graph launch
runs them all, with the host reading the energies once per block.

``sweep_cases`` draws the instances of the sweep workload: species uniform
over SPECIES and each coupling (t0-t3, x0-x3, W0; W0 moves b4p with it)
scaled by an independent uniform factor in [1 - rel, 1 + rel].

    python -m hfb.batch [--instances 256] [--workers 16] [--seed 20261203] [--graph --group 32]
"""
import argparse
import json
import threading
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import torch

from . import config, static
from .adjoint import force_overrides, theta_of

# name -> (N, Z, states per isospin, grid points per axis, spacing in fm)
SPECIES = {
    "O16": (8, 8, (10, 10), 24, 1.0),
    "Ca40": (20, 20, (24, 24), 32, 0.8),
    "Ca48": (28, 20, (34, 24), 32, 0.8),
    "Ni56": (28, 28, (34, 34), 32, 0.8),
    "Zr90": (50, 40, (60, 48), 40, 0.8),
    "Sn132": (82, 50, (90, 60), 40, 0.8),
}
SWEPT = ("t0", "t1", "t2", "t3", "x0", "x1", "x2", "x3", "W0")


def species_case(name):
    """Case dict of one species: SLy4 without pairing (all six are closed
    shells), oscillator start, x0 = 0.2, E0 = 100 MeV."""
    nn, nz, npsi, n, d = SPECIES[name]
    case = config.case_dict("O16")
    case["grid"] = dict(nx=n, ny=n, nz=n, dx=d, dy=d, dz=d)
    case["levels"] = dict(nneut=nn, nprot=nz, npsi=list(npsi))
    case["static"] = dict(maxiter=1500, serr=1e-20, x0dmp=0.2, e0dmp=100.0, tvaryx_0=True)
    rx, ry, rz = config.ho_radii(nn, nz)
    case["static"].update(radinx=rx, radiny=ry, radinz=rz)
    return case


def sweep_cases(instances=256, seed=20261203, rel=0.02, species=None):
    """[(species, case, factors)] for the sweep: species drawn uniformly,
    couplings scaled by independent U(1 - rel, 1 + rel) factors."""
    from .forces import init_forces
    rng = np.random.default_rng(seed)
    names = list(species or SPECIES)
    base = theta_of(init_forces(None, name="SLy4"))
    out = []
    for _ in range(instances):
        sp = names[int(rng.integers(len(names)))]
        f = rng.uniform(1.0 - rel, 1.0 + rel, len(SWEPT))
        theta = {k: base[k] * float(v) for k, v in zip(SWEPT, f)}
        out.append((sp, force_overrides(species_case(sp), theta), dict(zip(SWEPT, f.tolist()))))
    return out


def run_one(case, maxiter=1500):
    """Mixed-precision solve of one case on the current CUDA stream."""
    t0 = time.perf_counter()
    st = config.setup(case, dtype=torch.complex64)
    hist, sw = static.statichf_mixed(st, maxiter=maxiter)
    res = dict(ehf=hist[-1][1], iterations=len(hist), switch_iteration=sw,
               seconds=time.perf_counter() - t0)
    del st
    return res


def run_sweep(cases, workers=8, maxiter=1500):
    """Solve every case, ``workers`` at a time, each worker thread on its
    own CUDA stream.  Returns the results in the order of ``cases``."""
    local = threading.local()

    def job(k):
        if not hasattr(local, "stream"):
            local.stream = torch.cuda.Stream()
        with torch.cuda.stream(local.stream):
            r = run_one(cases[k][1], maxiter=maxiter)
            local.stream.synchronize()
        r["species"] = cases[k][0]
        return r

    if workers <= 1:
        return [job(k) for k in range(len(cases))]
    with ThreadPoolExecutor(max_workers=workers) as ex:
        return list(ex.map(job, range(len(cases))))


def run_sweep_graph(cases, group=32, maxiter=1500, block=10):
    """Solve every case with the graph driver, ``group`` instances per
    graph (the groups one after the other).  Results in case order."""
    from . import graph
    out = []
    for g0 in range(0, len(cases), group):
        chunk = cases[g0:g0 + group]
        t0 = time.perf_counter()
        states = [config.setup(c[1], dtype=torch.complex64) for c in chunk]
        res = graph.solve(states, maxiter=maxiter, block=block)
        dt = time.perf_counter() - t0
        for c, r in zip(chunk, res):
            out.append(dict(species=c[0], ehf=r["E"][-1], iterations=r["iterations"],
                            switch_iteration=r["switch"], seconds=dt))
        del states, res
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m hfb.batch")
    ap.add_argument("--instances", type=int, default=256)
    ap.add_argument("--workers", type=int, default=16)
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--maxiter", type=int, default=1500)
    ap.add_argument("--graph", action="store_true", help="graph driver: groups of instances per CUDA graph")
    ap.add_argument("--group", type=int, default=32)
    args = ap.parse_args(argv)
    cases = sweep_cases(args.instances, args.seed)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    if args.graph:
        res = run_sweep_graph(cases, group=args.group, maxiter=args.maxiter)
    else:
        res = run_sweep(cases, workers=args.workers, maxiter=args.maxiter)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    counts = {}
    for r in res:
        counts[r["species"]] = counts.get(r["species"], 0) + 1
    print(json.dumps(dict(op="sweep", instances=len(res), workers=args.workers, graph=args.graph,
                          group=args.group if args.graph else None, seconds=dt,
                          instances_per_second=len(res) / dt, species=counts,
                          iterations=int(sum(r["iterations"] for r in res)))), flush=True)


if __name__ == "__main__":
    main()
