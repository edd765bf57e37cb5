"""Spectral derivatives and the k-space preconditioner (oracle; test infrastructure).

Follows reference levels.py:132-437.  ``axis`` is the array axis of the spatial
direction (for a spinor ``(2, nx, ny, nz)`` the x axis is 1).
"""
import numpy as np


def _along(vec, axis, ndim):
    shp = [1] * ndim
    shp[axis] = vec.shape[0]
    return vec.reshape(shp)


def first_derivative_factors(n, d):
    """i*k*kfac/n with the k=0 and Nyquist entries zero (levels.py:139-146)."""
    kfac = 2.0 * np.pi / (d * n)
    half = n // 2
    m = np.zeros(n, dtype=np.complex128)
    q = np.arange(1, half)
    m[q] = 1j * q * kfac / n
    m[n - q] = -(1j * q * kfac) / n
    return m


def second_derivative_factors(n, d):
    """-(k*kfac)^2/n with the Nyquist entry kept at k=n/2 (levels.py:198-203)."""
    kfac = 2.0 * np.pi / (d * n)
    m = np.arange(n)
    k = np.minimum(m, n - m)
    return -(k * kfac) ** 2 / n


def cderv00(d, psin, axis):
    """First derivative, Nyquist zeroed (levels.py:132-189)."""
    n = psin.shape[axis]
    f = np.fft.fft(psin, axis=axis)
    f = f * _along(first_derivative_factors(n, d), axis, psin.ndim)
    return np.fft.ifft(f, axis=axis, norm="forward")


def cderv01(d, psin, axis):
    """First and second derivatives (levels.py:191-281)."""
    n = psin.shape[axis]
    f = np.fft.fft(psin, axis=axis)
    d1 = np.fft.ifft(f * _along(first_derivative_factors(n, d), axis, psin.ndim), axis=axis, norm="forward")
    d2 = np.fft.ifft(f * _along(second_derivative_factors(n, d), axis, psin.ndim), axis=axis, norm="forward")
    return d1, d2


def cderv02(d, psin, bfield, axis, spatial_axis):
    """d/dx psi and d/dx (B d/dx psi) (levels.py:284-395).

    ``bfield`` has the spatial shape ``(nx, ny, nz)``; ``spatial_axis`` is the
    direction (0, 1, 2) so the mean of B along it can be taken
    (levels.py:314-315).  The Nyquist bin of the second set is replaced by
    -(pi/d)^2 * mean(B) * psi_hat(Nyquist) / n.
    """
    n = psin.shape[axis]
    half = n // 2
    f = np.fft.fft(psin, axis=axis)
    nyq_in = np.take(f, half, axis=axis)
    d1 = np.fft.ifft(f * _along(first_derivative_factors(n, d), axis, psin.ndim), axis=axis, norm="forward")
    g = np.fft.fft(d1 * bfield, axis=axis)
    m = first_derivative_factors(n, d)
    g = g * _along(m, axis, psin.ndim)
    bmean = np.mean(bfield, axis=spatial_axis)
    nyq = -(np.pi / d) ** 2 * bmean * nyq_in / n
    idx = [slice(None)] * psin.ndim
    idx[axis] = half
    g[tuple(idx)] = nyq
    d2 = np.fft.ifft(g, axis=axis, norm="forward")
    return d1, d2


def k2_total(grids):
    """-(k_x^2 + k_y^2 + k_z^2) on the FFT grid, Nyquist included (levels.py:403-420)."""
    out = 0.0
    for a, (n, d) in enumerate(zip(grids.n, grids.d)):
        kfac = 2.0 * np.pi / (d * n)
        m = np.arange(n)
        k = np.minimum(m, n - m)
        out = out + _along(-(k * kfac) ** 2, a, 3)
    return out


def laplace(grids, h2ma, wg, wguv, psin, v_pairmax, e0inv):
    """(E0 + T)^-1 preconditioner in k space (levels.py:398-437).

    ``psin`` is one spinor ``(2, nx, ny, nz)``."""
    weight = max(wg, 0.1)
    weightuv = max(wguv, 0.1)
    ntot = grids.nx * grids.ny * grids.nz
    denom = (weight * (e0inv - h2ma * k2_total(grids)) + 0.5 * weightuv * v_pairmax) * ntot
    f = np.fft.fftn(psin, axes=(-3, -2, -1))
    f = f / denom
    return np.fft.ifftn(f, axes=(-3, -2, -1), norm="forward")
