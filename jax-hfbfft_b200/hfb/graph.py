"""Self-consistent iterations replayed as CUDA graphs, for one instance or
many instances in one graph launch.

In the steady state of the loop (past the BCS and diagonalisation start-up
phases of static.py:1755-1790 and the constant gap of pairs.py:143-157) the
device work of an iteration is the same sequence of library launches every
time, except for the step size x0dmp, which the step-control kernel
(hfb_step_control) now keeps on the device together with a history of
E_bind.  A block of iterations -- an even number, because the
diagonalisation step alternates between the state buffer and its spare --
is captured once into a CUDA graph per instance and replayed; the host
reads the energy history once per replay.  Several instances (different
nuclei, grids, couplings) are advanced by one launch of a composite graph
whose nodes are copies of the instances' captures (no edges between them,
so they run as concurrent branches); when instances finish or switch
precision the composite is rebuilt from the captures at hand, and only the
instance that switched is captured again.

Requirements of a replay: every scratch buffer of the library has reached
its size (the warm-up iterations do that, and a slot never shrinks), no
constraints and no configuration-space sub-iterations, and the precision of
an instance does not change inside a captured block.
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
        self.graph = None          # this run's captured block of iterations
        self.graph_block = None
        self.graph_dtype = None

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

    def capture(self, block):
        """Capture ``block`` iterations with device step control into this
        run's own graph (capture only records: the counters restart)."""
        self.to_device_control()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        i0 = self.i
        with torch.cuda.graph(g, capture_error_mode="relaxed"):
            for _ in range(block):
                self.record()
        self.i = i0
        self.count.zero_()
        self.read = 0
        torch.cuda.synchronize()
        self.graph, self.graph_block, self.graph_dtype = g, block, self.st["levels"].psi.dtype
        return g

    def drop_graph(self):
        """Back to ordinary iterations: the capture goes, the step size and
        previous values return to the host."""
        self.graph = None
        self.release_device_control()

    def release_device_control(self):
        """Back to host control: the step size and previous values from the device."""
        v = self.ctl.cpu().tolist()
        st, en = self.S["static"], self.S["energies"]
        st.x0dmp, en.ehfprev, en.efluct1prev, en.efluct2prev = v[0], v[1], v[2], v[3]
        st.x0_dev = None
        en.sync()


def _cuda_ok(res, what):
    err = res[0] if isinstance(res, tuple) else res
    if int(err) != 0:
        raise RuntimeError(f"{what}: CUDA error {int(err)}")
    return res[1] if isinstance(res, tuple) and len(res) > 1 else None


class _Composite:
    """One executable graph whose nodes are copies of several captured
    graphs, with no edges between them: one launch runs them all, as
    concurrent branches."""

    def __init__(self, graphs):
        from cuda.bindings import runtime as rt
        self.rt = rt
        self.graph = _cuda_ok(rt.cudaGraphCreate(0), "cudaGraphCreate")
        self.exe = None
        try:
            for g in graphs:
                child = rt.cudaGraph_t(init_value=g.raw_cuda_graph())
                _cuda_ok(rt.cudaGraphAddChildGraphNode(self.graph, None, 0, child), "cudaGraphAddChildGraphNode")
            self.exe = _cuda_ok(rt.cudaGraphInstantiate(self.graph, 0), "cudaGraphInstantiate")
        except Exception:
            self.close()
            raise

    def launch(self):
        st = self.rt.cudaStream_t(init_value=torch.cuda.current_stream().cuda_stream)
        _cuda_ok(self.rt.cudaGraphLaunch(self.exe, st), "cudaGraphLaunch")

    def close(self):
        if self.exe is not None:
            self.rt.cudaGraphExecDestroy(self.exe)
            self.exe = None
        if self.graph is not None:
            self.rt.cudaGraphDestroy(self.graph)
            self.graph = None


class BatchGraph:
    """Blocks of iterations of several GraphRuns advanced by one graph
    launch.  Each run's block is captured once into its own graph (again
    only when its precision changes), and the batch is the composite of
    those graphs: when instances finish or switch, the batch is recomposed
    from the captures it already has instead of recapturing every
    instance."""

    def __init__(self, runs, block=10):
        if block % 2:
            raise ValueError("block must be even (the diagonalisation step alternates two state buffers)")
        self.runs = list(runs)
        self.block = block
        self.comp = None
        self.streams = None

    def capture(self):
        for r in self.runs:
            if r.graph is None or r.graph_block != self.block or r.graph_dtype != r.st["levels"].psi.dtype:
                r.capture(self.block)
        try:
            self.comp = _Composite([r.graph for r in self.runs])
        except (ImportError, RuntimeError):
            # without the composite: each run's graph on a stream of its own
            self.comp = None
            self.streams = [torch.cuda.Stream() for _ in self.runs]
        return self

    def replay(self):
        """Advance every instance by one block of iterations."""
        if self.comp is not None:
            self.comp.launch()
        else:
            cur = torch.cuda.current_stream()
            for r, s in zip(self.runs, self.streams):
                s.wait_stream(cur)
                with torch.cuda.stream(s):
                    r.graph.replay()
            for s in self.streams:
                cur.wait_stream(s)
        for r in self.runs:
            r.i += self.block
        torch.cuda.synchronize()
        for r in self.runs:
            r.collect()

    def release(self):
        """Drop the composite; the runs keep their captures and device control."""
        if self.comp is not None:
            self.comp.close()
            self.comp = None


def solve(states, switch_mev=1e-3, stop_mev=5e-5, floor_mev=5e-5, maxiter=4000, block=10, graph_min=60,
          on_block=None, tune=True, fp32_min_points=static.FP32_MIN_POINTS):
    """Mixed-precision solves of several instances (states with complex64
    psi from hfb.config.setup) advanced together: ordinary iterations
    through the start-up phases, then graph replays of ``block`` iterations
    of every active instance per launch.  Each instance follows the
    precision rule of hfb.static.statichf_mixed (FP32 until the estimated
    remaining change is below ``switch_mev`` or the FP32 noise floor is
    reached, then FP64 until it is below ``stop_mev``); an instance's block
    is captured again only when it switches precision, and the batch graph
    is recomposed from the captures whenever an instance switches or
    finishes.  Problems smaller than ``fp32_min_points`` (states times grid
    points) run in FP64 throughout.  With ``tune``
    the single-precision hpsi kernel of each instance is chosen by
    measurement (hfb.tune, cached per grid and state count).  Returns one
    dict per instance: energies, the precision switch iteration, iterations
    and the hpsi kernel used."""
    from . import tune as _tune
    for s in states:
        if s["levels"].psi.dtype != torch.complex128 and s["levels"].nstmax * s["grids"].n3 < fp32_min_points:
            static.to_precision(s, torch.complex128)
    runs = [GraphRun(s) for s in states]
    info = [dict(switch=None if s["levels"].psi.dtype != torch.complex128 else 0, done=False,
                 prec="f32" if s["levels"].psi.dtype != torch.complex128 else "f64", hpsi=None) for s in states]
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
                r.drop_graph()
                active.remove(k)
            elif inf["prec"] == "f64" and r.st["levels"].psi.dtype != torch.complex128:
                r.drop_graph()
                static.to_precision(r.st, torch.complex128)
                tail_start[k] = len(r.E) - 1
                # the FP64 arrays are new: ordinary iterations grow the
                # library's scratch for them before the next capture
                r.plain(2)
    return [dict(E=r.E, switch=inf["switch"], iterations=r.i, state=r.st, hpsi=inf["hpsi"])
            for r, inf in zip(runs, info)]
