"""B200 (sm_100a) implementation of the static Skyrme HF+BCS iteration of
jax-hfbfft, behind the reference's module surface.

    import hfb
    st = hfb.config.setup(hfb.config.case_dict("O16"))
    out, res = hfb.static.statichf(**st)

Modules mirror the reference: params, forces, grids, levels, meanfield,
densities, coulomb, pairs, energies, inout, static, output.  Every array
operation runs in libhfb.so (CUDA, sm_100a) through the C ABI declared in
include/hfb.h; importing works without a GPU, computing does not.
"""
from . import _lib  # noqa: F401
from . import params, forces, grids, levels, meanfield, densities, coulomb, pairs, energies, inout  # noqa: F401
from . import static, output, config, adjoint, batch, restart, constraint  # noqa: F401

__version__ = "0.1.0"
