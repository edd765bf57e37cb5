"""Kernel-level timing on the bench workloads (also the small-case driver for
profiler captures).

    python -m hfb.microbench hpsi    [--case Pb208] [--states S] [--prec f32|f64] [--reps R]
    python -m hfb.microbench gram    [--case Pb208] [--prec f32|f64] [--reps R]
    python -m hfb.microbench iterate [--case Pb208] [--prec f32|f64] [--reps R] [--skip N]
    python -m hfb.microbench kernels [--case Pb208] [--prec f32|f64] [--reps R] [--skip N] [--top K]

Every mode builds the workload's oscillator start and its mean field
(``static.prepare``), runs the operation ``--warmup`` times and then ``--reps``
times between CUDA events on the launching stream, and prints one JSON line
with the mean time per call; the timed calls run inside an NVTX range
"timed" (``ncu --nvtx --nvtx-include timed/``).  ``--states`` limits hpsi to the first S states
(the potentials stay those of the full nucleus), which keeps a profiler
capture small.
"""
import argparse
import json
import os
import sys

import torch

from . import config, static
from ._lib import call, ptr, stream_ptr, prec_of


def _setup(case, dtype):
    st = config.setup(config.case_dict(case), dtype=dtype)
    S = {k: st[k] for k in static._STATE_KEYS}
    static.prepare(**S)
    torch.cuda.synchronize()
    return st, S


def _time(fn, warmup, reps):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    s = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("timed")   # lets a profiler select exactly these launches
    e0.record(s)
    for _ in range(reps):
        fn()
    e1.record(s)
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3 / max(reps, 1)


def run_hpsi(args, dtype):
    st, _ = _setup(args.case, dtype)
    lv, mf, g = st["levels"], st["meanfield"], st["grids"]
    ns = args.states if args.states > 0 else lv.nstmax
    nn = min(ns, lv.npsi[0])
    psi = lv.psi[:ns].contiguous()
    mf.pack(dtype)
    out = torch.empty_like(psi)
    wt = torch.ones(ns, dtype=torch.float64, device="cuda")
    wu = torch.zeros(ns, dtype=torch.float64, device="cuda")

    def once():
        call("hfb_hpsi", g.ctx.handle, prec_of(psi), ptr(mf.pot), ns, nn, ptr(psi), ptr(wt), ptr(wu), None,
             ptr(out), None, stream_ptr())

    t = _time(once, args.warmup, args.reps)
    n3 = g.n3
    esz = psi.element_size()
    alg = ns * 4 * n3 * esz + 2 * 12 * n3 * (esz // 2)
    return dict(op="hpsi", states=ns, seconds=t, algorithmic_bytes=alg, gbs=alg / t / 1e9)


def run_gram(args, dtype):
    st, _ = _setup(args.case, dtype)
    lv, g = st["levels"], st["grids"]
    n0, n1 = lv.npsi
    ns = n0 + n1
    psi = lv.psi
    hp = torch.empty_like(psi).copy_(psi)
    out = torch.zeros((4, n0, n0), dtype=torch.complex128, device="cuda")
    vp = torch.ones(g.n3, dtype=torch.float64, device="cuda")

    def once():
        call("hfb_gram", g.ctx.handle, prec_of(psi), 0, n0, 15, ptr(psi), ptr(hp), ptr(hp), ptr(vp), g.wxyz,
             ptr(out), stream_ptr())

    t = _time(once, args.warmup, args.reps)
    K = 2 * g.n3
    flops = 4 * 8.0 * n0 * n0 * K
    return dict(op="gram", states=n0, matrices=4, seconds=t, complex_flops=flops, tflops=flops / t / 1e12)


def run_iterate(args, dtype):
    st, S = _setup(args.case, dtype)
    it = [0]

    def once():
        it[0] += 1
        static.iterate(it[0], **S)

    from ._lib import launch_count
    l0 = launch_count()
    for _ in range(args.skip):
        once()
    l1 = launch_count()
    t = _time(once, args.warmup, args.reps)
    l2 = launch_count()
    return dict(op="iterate", seconds=t, energy=st["energies"].ehf, first_timed_iteration=args.skip + args.warmup + 1,
                launches_before_timed=l1 + (l2 - l1) * args.warmup // (args.warmup + args.reps),
                launches_setup=l0, launches_per_iteration=(l2 - l1) / (args.warmup + args.reps))


def run_kernels(args, dtype):
    """Per-kernel device time of ``--reps`` iterations after the untimed
    ones, from the CUDA activity trace of torch.profiler (kernels overlap
    as in an ordinary run; the trace adds host-side overhead only)."""
    from torch.profiler import profile, ProfilerActivity
    st, S = _setup(args.case, dtype)
    i = 0
    for _ in range(args.skip + args.warmup):
        i += 1
        static.iterate(i, **S)
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        for _ in range(args.reps):
            i += 1
            static.iterate(i, **S)
        torch.cuda.synchronize()
    rows = []
    for e in prof.key_averages():
        t = getattr(e, "device_time_total", None)
        if t is None:
            t = getattr(e, "cuda_time_total", 0.0)
        if t > 0:
            rows.append((t, e.count, e.key))
    rows.sort(reverse=True)
    tot = sum(r[0] for r in rows)
    top = [dict(kernel=k[:90], calls_per_iteration=c / args.reps, us_per_iteration=t / args.reps,
                share=t / tot) for t, c, k in rows[:args.top]]
    return dict(op="kernels", us_per_iteration_total=tot / args.reps, kernels=top)


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m hfb.microbench")
    ap.add_argument("op", choices=("hpsi", "gram", "iterate", "kernels"))
    ap.add_argument("--case", default="Pb208")
    ap.add_argument("--prec", default="f32", choices=("f32", "f64"))
    ap.add_argument("--states", type=int, default=0)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--skip", type=int, default=0, help="iterate: untimed iterations before the warm-up")
    ap.add_argument("--top", type=int, default=25, help="kernels: rows to print")
    args = ap.parse_args(argv)
    dtype = torch.complex64 if args.prec == "f32" else torch.complex128
    fn = {"hpsi": run_hpsi, "gram": run_gram, "iterate": run_iterate, "kernels": run_kernels}[args.op]
    res = fn(args, dtype)
    res.update(case=args.case, prec=args.prec, reps=args.reps)
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
