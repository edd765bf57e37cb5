"""Coulomb potential by FFT on a doubled grid (oracle; test infrastructure).

Follows reference coulomb.py:14-75.
"""
from dataclasses import dataclass
import numpy as np

from .model import E2


@dataclass
class Coulomb:
    nx2: int
    ny2: int
    nz2: int
    wcoul: np.ndarray
    q: np.ndarray


def _iq(n, d, periodic):
    """coulomb.py:14-21: squared distances (or squared k) on the wrapped index."""
    i = np.arange(n)
    i = np.where(i <= n // 2, i, i - n)
    if periodic:
        return (2.0 * np.pi * i / (n * d)) ** 2
    return (d * i) ** 2


def init_coulomb(grids):
    """Green's function of 1/r on the (2n)^3 grid (coulomb.py:23-52).
    The r=0 cell holds 2.84 / dV^(1/3)."""
    nx2 = grids.nx if grids.periodic else 2 * grids.nx
    ny2 = grids.ny if grids.periodic else 2 * grids.ny
    nz2 = grids.nz if grids.periodic else 2 * grids.nz
    q = (_iq(nx2, grids.dx, grids.periodic)[:, None, None] + _iq(ny2, grids.dy, grids.periodic)[None, :, None]
         + _iq(nz2, grids.dz, grids.periodic)[None, None, :]).astype(np.complex128)
    q[0, 0, 0] = 1.0
    if grids.periodic:
        q = 1.0 / q.real
        q[0, 0, 0] = 0.0
        q = q.astype(np.complex128)
    else:
        q = 1.0 / np.sqrt(q.real)
        q[0, 0, 0] = 2.84 / (grids.dx * grids.dy * grids.dz) ** (1.0 / 3.0)
        q = np.fft.fftn(q)
    return Coulomb(nx2=nx2, ny2=ny2, nz2=nz2, wcoul=np.zeros((grids.nx, grids.ny, grids.nz)), q=q)


def poisson(grids, coulomb, rho):
    """Coulomb potential of the proton density rho[1] (coulomb.py:54-75)."""
    r2 = np.zeros((coulomb.nx2, coulomb.ny2, coulomb.nz2), dtype=np.complex128)
    r2[:grids.nx, :grids.ny, :grids.nz] = rho[1]
    r2 = np.fft.fftn(r2)
    if grids.periodic:
        r2 = r2 * (4.0 * np.pi * E2 * np.real(coulomb.q))
    else:
        r2 = r2 * (E2 * grids.wxyz * coulomb.q)
    w = np.fft.ifftn(r2)
    return np.real(w[:grids.nx, :grids.ny, :grids.nz])
