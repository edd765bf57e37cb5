"""CPU FP64 oracle for the static Skyrme HF+BCS iteration of jax-hfbfft.

TEST INFRASTRUCTURE ONLY.  This package is a NumPy/SciPy restatement of the
reference's algorithm (every function cites the reference file:line it
follows).  It is the checker for the CUDA path: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` may import it.  The product (``jax-hfbfft_b200/hfb``)
never imports, links or executes anything from here.

Parity pin: the restatement is checked against golden vectors that were
produced by executing the reference modules themselves (unmodified) under a
NumPy-backed stand-in for the subset of the ``jax`` API they use, because JAX
is not installable in the build container (``tests/golden/make_golden.py``).

Modules
-------
model      constants, Skyrme force table, grids, derived coefficients, levels
spectral   FFT derivatives (cderv*00/01/02) and the k-space preconditioner
meanfield  hpsi01 and the skyrme potential builder
densities  add_density
coulomb    init_coulomb / poisson (doubled-grid FFT)
pairs      BCS gap / Fermi level / occupations
static     harmosc, grstep, diagstep, the iteration driver
energies   integ_energy, sum_energy, sp_properties, rms radii
"""
from . import model, spectral, meanfield, densities, coulomb, pairs, static, energies  # noqa: F401
