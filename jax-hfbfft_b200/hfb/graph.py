"""Self-consistent iterations replayed as CUDA graphs, for one instance or
many instances in one graph launch.

In the steady state of the loop (past the BCS and diagonalisation start-up
phases of static.py:1755-1790 and the constant gap of pairs.py:143-157) the
device work of an iteration is the same sequence of library launches every
time, except for the step size x0dmp, which the step-control kernel
(hfb_step_control) now keeps on the device together with a history of
E_bind.  A block of iterations -- an even number, because the
diagonalisation step alternates between the state buffer and its spare --
is captured once into a CUDA graph and replayed; the host reads the energy
history once per replay.  Several instances (different nuclei, grids,
couplings) are captured into the same graph, each on its own stream forked
from the capture stream, so one graph launch advances all of them.

Requirements of a replay: every scratch buffer of the library has reached
its size (the warm-up iterations do that, and a slot never shrinks), no
constraints and no configuration-space sub-iterations, and the precision of
an instance does not change inside a captured block (the mixed driver
recaptures when an instance switches to FP64).
"""
import ctypes as C

import torch

from . import static
from ._lib import call, ptr, stream_ptr

_E_BIND = 12   # index of ehf in Energies.dev (hfb._lib.ENERGY_KEYS)


class GraphRun:
    """One instance (a state dict from hfb.config.setup) driven by graph
    replays after ``warm`` ordinary iterations."""

    def __init__(self, state, max_hist=20000):
        self.st = state
        self.S = {k: state[k] for k in static._STATE_KEYS}
        self.ctl = torch.zeros(6, dtype=torch.float64, device="cuda")
        self.hist = torch.zeros(max_hist, dtype=torch.float64, device="cuda")
        self.count = torch.zeros(1, dtype=torch.int32, device="cuda")
        self.max_hist = max_hist
        self.i = 0                 # last iteration done
        self.read = 0              # history entries already read by the host
        self.E = []                # E_bind per iteration (host copy)
        self.prepared = False

    def steady_from(self):
        """First iteration index whose device work no longer depends on it."""
        st = self.S["static"]
        return max(st.inibcs, st.inidiag, 10) + 2

    def start(self):
        static.prepare(**self.S)
        self.S["energies"].sync()
        self.prepared = True

    def plain(self, n):
        """``n`` ordinary iterations (host step-size control)."""
        for _ in range(n):
            self.i += 1
            static.iterate(self.i, **self.S)
            self.E.append(self.S["energies"].ehf)

    def to_device_control(self):
        """Move the step size and the adaptation's previous values to the
        device; the gradient step reads the step size from there."""
        st, en = self.S["static"], self.S["energies"]
        vals = [st.x0dmp, en.ehfprev, en.efluct1prev, en.efluct2prev, st.x0dmpmin, 1.0 if st.tvaryx_0 else 0.0]
        self.ctl.copy_(torch.tensor(vals, dtype=torch.float64))
        st.x0_dev = self.ctl[0:1]
        self.count.zero_()
        self.read = 0

    def record(self):
        """The device work of the next iteration, then step control."""
        self.i += 1
        static.iterate_device(self.i, **self.S)
        en = self.S["energies"]
        call("hfb_step_control", self.S["grids"].ctx.handle, ptr(en.dev[_E_BIND:_E_BIND + 1]), ptr(en.efluct_dev),
             ptr(self.ctl), ptr(self.hist), ptr(self.count), self.max_hist, stream_ptr())

    def collect(self):
        """Copy the new history entries to the host (after a replay)."""
        n = int(self.count.item())
        if n > self.read:
            self.E.extend(self.hist[self.read:n].cpu().tolist())
            self.read = n
        self.S["grids"].ctx.check(f"graph replay up to iteration {self.i}")

    def release_device_control(self):
        """Back to host control: the step size and previous values from the device."""
        v = self.ctl.cpu().tolist()
        st, en = self.S["static"], self.S["energies"]
        st.x0dmp, en.ehfprev, en.efluct1prev, en.efluct2prev = v[0], v[1], v[2], v[3]
        st.x0_dev = None
        en.sync()


class BatchGraph:
    """Captured blocks of iterations of several GraphRuns in one CUDA graph."""

    def __init__(self, runs, block=10):
        if block % 2:
            raise ValueError("block must be even (the diagonalisation step alternates two state buffers)")
        self.runs = list(runs)
        self.block = block
        self.graph = None
        self.base = [r.i for r in self.runs]

    def capture(self):
        for r in self.runs:
            r.to_device_control()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        streams = [torch.cuda.Stream() for _ in self.runs]
        starts = [r.i for r in self.runs]
        with torch.cuda.graph(g, capture_error_mode="relaxed"):
            cur = torch.cuda.current_stream()
            for r, s in zip(self.runs, streams):
                s.wait_stream(cur)
                with torch.cuda.stream(s):
                    for _ in range(self.block):
                        r.record()
            for s in streams:
                cur.wait_stream(s)
        # capture only recorded the work: the iteration counters restart
        for r, i0 in zip(self.runs, starts):
            r.i = i0
            r.count.zero_()
            r.read = 0
        self.graph = g
        self.streams = streams
        torch.cuda.synchronize()
        return self

    def replay(self):
        """Advance every instance by one block of iterations."""
        self.graph.replay()
        for r in self.runs:
            r.i += self.block
        torch.cuda.synchronize()
        for r in self.runs:
            r.collect()

    def release(self):
        for r in self.runs:
            r.release_device_control()
        self.graph = None


def solve(states, switch_mev=5e-4, stop_mev=5e-5, floor_mev=5e-5, maxiter=4000, block=10, graph_min=60,
          on_block=None, tune=True):
    """Mixed-precision solves of several instances (states with complex64
    psi from hfb.config.setup) advanced together: ordinary iterations
    through the start-up phases, then graph replays of ``block`` iterations
    of every active instance per launch.  Each instance follows the
    precision rule of hfb.static.statichf_mixed (FP32 until the estimated
    remaining change is below ``switch_mev`` or the FP32 noise floor is
    reached, then FP64 until it is below ``stop_mev``); the graph is
    recaptured whenever an instance switches or finishes.  With ``tune``
    the single-precision hpsi kernel of each instance is chosen by
    measurement (hfb.tune, cached per grid and state count).  Returns one
    dict per instance: energies, the precision switch iteration, iterations
    and the hpsi kernel used."""
    from . import tune as _tune
    runs = [GraphRun(s) for s in states]
    info = [dict(switch=None, done=False, prec="f32", hpsi=None) for _ in runs]
    for r, inf in zip(runs, info):
        r.start()
        if tune:
            inf["hpsi"] = _tune.tune_hpsi(r.st)
        r.plain(max(r.steady_from(), 2))
    active = list(range(len(runs)))
    tail_start = [None] * len(runs)
    while active:
        bg = BatchGraph([runs[k] for k in active], block=block).capture()
        changed = False
        while not changed:
            bg.replay()
            if on_block is not None:
                on_block([runs[k] for k in active])
            for k in active:
                r, inf = runs[k], info[k]
                E = r.E if inf["prec"] == "f32" else r.E[tail_start[k]:]
                rem = static.remaining_change(E)
                if r.i >= maxiter:
                    inf["done"] = changed = True
                elif inf["prec"] == "f32":
                    recent = [abs(E[j] - E[j - 1]) for j in range(max(1, len(E) - 25), len(E))]
                    if (rem is not None and abs(rem) < switch_mev) or (len(E) > graph_min and max(recent) < floor_mev):
                        inf["prec"], inf["switch"], changed = "f64", r.i, True
                elif len(E) >= 3 and rem is not None and abs(rem) < stop_mev:
                    inf["done"] = changed = True
        bg.release()
        for k in list(active):
            r, inf = runs[k], info[k]
            if inf["done"]:
                active.remove(k)
            elif inf["prec"] == "f64" and r.st["levels"].psi.dtype != torch.complex128:
                static.to_precision(r.st, torch.complex128)
                tail_start[k] = len(r.E) - 1
                # the FP64 arrays are new: ordinary iterations grow the
                # library's scratch for them before the next capture
                r.plain(2)
    return [dict(E=r.E, switch=inf["switch"], iterations=r.i, state=r.st, hpsi=inf["hpsi"])
            for r, inf in zip(runs, info)]
