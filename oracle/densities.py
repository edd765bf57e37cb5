"""Occupation-weighted local densities (oracle; test infrastructure).

Follows reference densities.py:177-330 (the live ``add_density`` path; the
unused helper at densities.py:33-175 is not restated).
"""
from dataclasses import dataclass
import numpy as np

from . import pool
from .spectral import cderv00


@dataclass
class Densities:
    rho: np.ndarray      # (2, nx, ny, nz)
    chi: np.ndarray
    tau: np.ndarray
    current: np.ndarray  # (2, 3, nx, ny, nz)
    sdens: np.ndarray
    sodens: np.ndarray


def init_densities(grids):
    s4 = (2, grids.nx, grids.ny, grids.nz)
    s5 = (2, 3, grids.nx, grids.ny, grids.nz)
    return Densities(rho=np.zeros(s4), chi=np.zeros(s4), tau=np.zeros(s4), current=np.zeros(s5),
                     sdens=np.zeros(s5), sodens=np.zeros(s5))


def state_contributions(weight, weightuv, psin, d):
    """Per-state terms of compute_single_contribution (densities.py:237-330).

    ``psin`` is ``(nst, 2, nx, ny, nz)``; weights are ``(nst,)``.
    Returns ``rho, chi, tau (nst, ...)`` and ``current, sdens, sodens (nst, 3, ...)``.
    """
    w = weight[:, None, None, None]
    wu = weightuv[:, None, None, None]
    a = psin[:, 0]
    b = psin[:, 1]
    aa = (a * np.conj(a) + b * np.conj(b)).real
    rho = w * aa
    chi = 0.5 * wu * aa
    ab = np.conj(a) * b
    sdens = np.stack([2.0 * w * ab.real, 2.0 * w * ab.imag, w * (np.conj(a) * a - np.conj(b) * b).real], axis=1)
    dx = cderv00(d[0], psin, axis=2)
    dy = cderv00(d[1], psin, axis=3)
    dz = cderv00(d[2], psin, axis=4)
    tau = np.zeros_like(rho)
    cur = []
    for q in (dx, dy, dz):
        tau = tau + w * (q[:, 0] * np.conj(q[:, 0]) + q[:, 1] * np.conj(q[:, 1])).real
        cur.append(w * (q[:, 0] * np.conj(a) + q[:, 1] * np.conj(b)).imag)
    # spin-orbit density (densities.py:270-315)
    j_y_x = -w * (dx[:, 0] * np.conj(a) - dx[:, 1] * np.conj(b)).imag
    j_z_x = -w * (a * np.conj(dx[:, 1]) - b * np.conj(dx[:, 0])).real
    j_x_y = w * (dy[:, 0] * np.conj(a) - dy[:, 1] * np.conj(b)).imag
    j_z_y = -w * (dy[:, 1] * np.conj(a) + dy[:, 0] * np.conj(b)).imag
    j_x_z = w * (dz[:, 1] * np.conj(a) - dz[:, 0] * np.conj(b)).real
    j_y_z = w * (dz[:, 1] * np.conj(a) + dz[:, 0] * np.conj(b)).imag
    sodens = np.stack([j_x_y + j_x_z, j_y_x + j_y_z, j_z_x + j_z_y], axis=1)
    return rho, chi, tau, np.stack(cur, axis=1), sdens, sodens


def add_density(dens, grids, levels):
    """Sum the per-state terms by isospin (densities.py:177-234)."""
    weight = levels.wocc * levels.wstates
    weightuv = levels.wguv * levels.pairwg * levels.wstates
    out = {k: [] for k in ("rho", "chi", "tau", "current", "sdens", "sodens")}
    for iq in range(2):
        b = levels.block(iq)

        def part(sl):
            r = state_contributions(weight[sl], weightuv[sl], levels.psi[sl], grids.d)
            return [v.sum(axis=0) for v in r]

        parts = pool.pmap(part, pool.chunks(b.start, b.stop))
        for j, k in enumerate(out):
            acc = parts[0][j]
            for p in parts[1:]:
                acc = acc + p[j]
            out[k].append(acc)
    for k in out:
        setattr(dens, k, np.stack(out[k]))
    return dens
