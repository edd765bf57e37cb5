"""Host-thread parallelism for the oracle (test infrastructure).

The per-state work of an iteration (two Hamiltonian applications, the
preconditioner, the density terms, the single-particle properties) is
independent from state to state, and NumPy's array loops and FFTs release
the GIL on arrays of this size, so chunks of states run concurrently on
host threads.  With one worker (the default, used by every parity test)
each helper processes all states as one chunk, in the original order.

``set_workers(n)`` sets the thread count (``None`` or 0: ``os.cpu_count()``).
"""
import concurrent.futures as _cf
import os

_workers = 1
_executor = None


def set_workers(n):
    """Use ``n`` host threads for the per-state work (1 = serial)."""
    global _workers, _executor
    n = int(n) if n else (os.cpu_count() or 1)
    n = max(1, n)
    if n != _workers and _executor is not None:
        _executor.shutdown(wait=True)
        _executor = None
    _workers = n


def workers():
    return _workers


def chunks(start, stop):
    """Split the state range [start, stop) into at most ``workers()``
    contiguous slices of near-equal length."""
    n = stop - start
    k = max(1, min(_workers, n))
    out, s = [], start
    for c in range(k):
        e = s + n // k + (1 if c < n % k else 0)
        if e > s:
            out.append(slice(s, e))
        s = e
    return out


def pmap(fn, items):
    """``[fn(x) for x in items]``, on the worker threads when there are more
    than one."""
    global _executor
    items = list(items)
    if _workers <= 1 or len(items) <= 1:
        return [fn(x) for x in items]
    if _executor is None:
        _executor = _cf.ThreadPoolExecutor(_workers)
    return list(_executor.map(fn, items))
