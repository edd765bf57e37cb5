"""NumPy-backed stand-in for the subset of the ``jax`` API used by jax-hfbfft.

JAX is not installed in the build container and cannot be installed (no
network).  The golden-vector generator (``tests/golden/make_golden.py``) puts
this directory first on ``sys.path`` and then imports the reference modules
unmodified, so the reference's own code produces the golden vectors.

Semantics restated from the public JAX documentation:

* ``jax.jit`` / ``partial(jax.jit, static_argnames=...)``: tracing is dropped;
  the wrapped function runs eagerly (results are identical up to rounding
  because every op is evaluated in float64/complex128, x64 mode).
* ``jax.vmap``: a Python loop over the mapped axis, outputs stacked on axis 0.
* ``jax.lax.cond``: an eager ``if``.
* ``x.at[idx].set/add/multiply/divide``: functional updates returning a copy;
  out-of-bounds integer indices are dropped (JAX's default scatter mode).
* ``jax.ops.segment_sum``: ``np.add.at`` into ``num_segments`` rows.
* ``jnp.linalg.eigh(a, symmetrize_input=False)``: LAPACK ``heevd`` on the lower
  triangle (``UPLO='L'``), which is what JAX does on CPU.
* ``jnp.argsort``: stable sort (JAX's default).

This is test infrastructure only; nothing in the product imports it.
"""
import numpy as _np

from . import numpy  # noqa: F401  (jax.numpy)
from . import lax, tree_util, ops, profiler  # noqa: F401
from .numpy import JArray as Array  # noqa: F401


def jit(fun=None, **_kwargs):
    if fun is None:
        return lambda f: f
    return fun


def block_until_ready(x):
    return x


def vmap(fun, in_axes=0, out_axes=0):
    def mapped(*args):
        axes = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)
        n = None
        for a, ax in zip(args, axes):
            if ax is not None:
                n = _np.shape(a)[ax]
                break
        outs = []
        for i in range(n):
            call = [(_np.take(a, i, axis=ax) if ax is not None else a) for a, ax in zip(args, axes)]
            outs.append(fun(*call))
        if isinstance(outs[0], tuple):
            return tuple(numpy.stack([o[k] for o in outs]) for k in range(len(outs[0])))
        return numpy.stack(outs)
    return mapped


class _Config:
    def update(self, *_a, **_k):
        pass


config = _Config()
