"""Single-particle Hamiltonian and Skyrme potentials (oracle; test infrastructure).

Follows reference meanfield.py:7-391.
"""
from dataclasses import dataclass
import numpy as np

from .model import apply_along
from .spectral import cderv00, cderv02
from .coulomb import poisson


@dataclass
class Meanfield:
    upot: np.ndarray      # (2, nx, ny, nz)
    bmass: np.ndarray
    divaq: np.ndarray
    v_pair: np.ndarray
    aq: np.ndarray        # (2, 3, nx, ny, nz)
    spot: np.ndarray
    wlspot: np.ndarray
    dbmass: np.ndarray
    ecorrp: float = 0.0


def init_meanfield(grids):
    """meanfield.py:23-38."""
    s4 = (2, grids.nx, grids.ny, grids.nz)
    s5 = (2, 3, grids.nx, grids.ny, grids.nz)
    return Meanfield(upot=np.zeros(s4), bmass=np.zeros(s4), divaq=np.zeros(s4), v_pair=np.zeros(s4),
                     aq=np.zeros(s5), spot=np.zeros(s5), wlspot=np.zeros(s5), dbmass=np.zeros(s5))


def hpsi01(grids, mf, iq, weight, weightuv, pinn):
    """h_q applied to a 2-spinor (meanfield.py:41-159).

    ``pinn`` may carry leading batch axes: ``(..., 2, nx, ny, nz)``; ``weight``
    and ``weightuv`` are then broadcastable to the batch shape.
    Returns ``(pout, pout_mf, pout_del)``.
    """
    up = mf.upot[iq]
    bm = mf.bmass[iq]
    aq = mf.aq[iq]
    sp = mf.spot[iq]
    wl = mf.wlspot[iq]
    vp = mf.v_pair[iq]
    p0 = pinn[..., 0, :, :, :]
    p1 = pinn[..., 1, :, :, :]
    h = 0.5

    # local and spin-current terms (meanfield.py:47-58)
    o0 = up * p0 + (sp[0] - 1j * sp[1]) * p1 + sp[2] * p0
    o1 = up * p1 + (sp[0] + 1j * sp[1]) * p0 - sp[2] * p1

    # x (meanfield.py:60-87)
    d1, d2 = cderv02(grids.dx, pinn, bm, axis=-3, spatial_axis=0)
    o0 = o0 - 1j * (h * aq[0] - h * wl[1]) * d1[..., 0, :, :, :] - h * wl[2] * d1[..., 1, :, :, :] - d2[..., 0, :, :, :]
    o1 = o1 - 1j * (h * aq[0] + h * wl[1]) * d1[..., 1, :, :, :] + h * wl[2] * d1[..., 0, :, :, :] - d2[..., 1, :, :, :]
    w = np.stack([-0.5j * (aq[0] - wl[1]) * p0 - h * wl[2] * p1,
                  -0.5j * (aq[0] + wl[1]) * p1 + h * wl[2] * p0], axis=-4)
    c = cderv00(grids.dx, w, axis=-3)
    o0 = o0 + c[..., 0, :, :, :]
    o1 = o1 + c[..., 1, :, :, :]

    # y (meanfield.py:89-116)
    d1, d2 = cderv02(grids.dy, pinn, bm, axis=-2, spatial_axis=1)
    o0 = o0 - 1j * (h * aq[1] + h * wl[0]) * d1[..., 0, :, :, :] + 1j * (h * wl[2]) * d1[..., 1, :, :, :] - d2[..., 0, :, :, :]
    o1 = o1 - 1j * (h * aq[1] - h * wl[0]) * d1[..., 1, :, :, :] + 1j * (h * wl[2]) * d1[..., 0, :, :, :] - d2[..., 1, :, :, :]
    w = np.stack([-0.5j * (aq[1] + wl[0]) * p0 + 0.5j * wl[2] * p1,
                  -0.5j * (aq[1] - wl[0]) * p1 + 0.5j * wl[2] * p0], axis=-4)
    c = cderv00(grids.dy, w, axis=-2)
    o0 = o0 + c[..., 0, :, :, :]
    o1 = o1 + c[..., 1, :, :, :]

    # z (meanfield.py:118-145)
    d1, d2 = cderv02(grids.dz, pinn, bm, axis=-1, spatial_axis=2)
    o0 = o0 - 1j * (h * aq[2]) * d1[..., 0, :, :, :] + (h * wl[0] - 1j * (h * wl[1])) * d1[..., 1, :, :, :] - d2[..., 0, :, :, :]
    o1 = o1 - 1j * (h * aq[2]) * d1[..., 1, :, :, :] + (-h * wl[0] - 1j * (h * wl[1])) * d1[..., 0, :, :, :] - d2[..., 1, :, :, :]
    w = np.stack([-0.5j * aq[2] * p0 + (h * wl[0] - 0.5j * wl[1]) * p1,
                  -0.5j * aq[2] * p1 + (-h * wl[0] - 0.5j * wl[1]) * p0], axis=-4)
    c = cderv00(grids.dz, w, axis=-1)
    o0 = o0 + c[..., 0, :, :, :]
    o1 = o1 + c[..., 1, :, :, :]

    pout_mf = np.stack([o0, o1], axis=-4)
    pout_del = pinn * vp
    wt = np.asarray(weight, dtype=np.float64)
    wu = np.asarray(weightuv, dtype=np.float64)
    if wt.ndim:
        wt = wt.reshape(wt.shape + (1, 1, 1, 1))
    if wu.ndim:
        wu = wu.reshape(wu.shape + (1, 1, 1, 1))
    pout = wt * pout_mf - wu * pout_del
    return pout, pout_mf, pout_del


def _curl(grids, v):
    """curl of a (3, nx, ny, nz) field with the dense derivative matrices."""
    D = grids.der1
    return np.stack([apply_along(D[1], v[2], 1) - apply_along(D[2], v[1], 2),
                     apply_along(D[2], v[0], 2) - apply_along(D[0], v[2], 0),
                     apply_along(D[0], v[1], 0) - apply_along(D[1], v[0], 1)])


def skyrme(coulomb, dens, forces, grids, mf, tcoul=True):
    """Potentials from densities (meanfield.py:164-391).  Updates ``mf`` and
    ``coulomb.wcoul`` in place and returns them."""
    f = forces
    rho, tau, cur, sd, so, chi = dens.rho, dens.tau, dens.current, dens.sdens, dens.sodens, dens.chi
    D1, D2 = grids.der1, grids.der2
    rt = rho[0] + rho[1]
    rtp = rt ** f.power
    upot = np.zeros_like(rho)
    for iq in range(2):                                   # step 1 (181-190)
        ic = 1 - iq
        upot[iq] = rtp * ((f.b3 * (f.power + 2.0) / 3.0 - 2.0 * f.b3p / 3.0) * rho[iq]
                          + f.b3 * (f.power + 2.0) / 3.0 * rho[ic]
                          - (f.b3p * f.power / 3.0) * (rho[0] ** 2 + rho[1] ** 2) / (rt + 1.0e-25))
    divj = np.stack([sum(apply_along(D1[a], so[iq, a], a) for a in range(3)) for iq in range(2)])
    for iq in range(2):                                   # step 2 (195-206)
        upot[iq] += -(f.b4 + f.b4p) * divj[iq] - f.b4 * divj[1 - iq]
    if tcoul:                                             # step 3 (211-221)
        coulomb.wcoul = poisson(grids, coulomb, rho)
        upot[1] += coulomb.wcoul
        if f.ex != 0:
            upot[1] += -f.slate * rho[1] ** (1.0 / 3.0)
    lap = np.stack([sum(apply_along(D2[a], rho[iq], a) for a in range(3)) for iq in range(2)])
    for iq in range(2):                                   # step 4 (227-241)
        ic = 1 - iq
        upot[iq] += ((f.b0 - f.b0p) * rho[iq] + f.b0 * rho[ic] + (f.b1 - f.b1p) * tau[iq] + f.b1 * tau[ic]
                     - (f.b2 - f.b2p) * lap[iq] - f.b2 * lap[ic])
    bmass = np.stack([f.h2m[iq] + (f.b1 - f.b1p) * rho[iq] + f.b1 * rho[1 - iq] for iq in range(2)])  # step 5
    grad = np.stack([np.stack([apply_along(D1[a], rho[iq], a) for a in range(3)]) for iq in range(2)])
    wlspot = np.stack([(f.b4 + f.b4p) * grad[iq] + f.b4 * grad[1 - iq] for iq in range(2)])          # step 6
    cs = np.stack([_curl(grids, sd[iq]) for iq in range(2)])                                         # step 7
    aq = np.stack([-2.0 * (f.b1 - f.b1p) * cur[iq] - 2.0 * f.b1 * cur[1 - iq]
                   - (f.b4 + f.b4p) * cs[iq] - f.b4 * cs[1 - iq] for iq in range(2)])               # step 8
    cj = np.stack([_curl(grids, cur[iq]) for iq in range(2)])                                        # step 9
    spot = np.stack([-(f.b4 + f.b4p) * cj[iq] - f.b4 * cj[1 - iq] for iq in range(2)])               # step 10
    divaq = np.stack([sum(apply_along(D1[a], aq[iq, a], a) for a in range(3)) for iq in range(2)])   # step 11
    dbmass = np.stack([np.stack([apply_along(D1[a], bmass[iq], a) for a in range(3)]) for iq in range(2)])
    if f.ipair == 6:                                      # step 13 (352-366)
        rearr = (f.v0neut / f.rho0pr) * chi[0] ** 2 + (f.v0prot / f.rho0pr) * chi[1] ** 2
        upot[0] += rearr
        upot[1] += rearr
        mf.ecorrp = -np.sum(rt * rearr) * grids.wxyz / 2.0
    else:
        mf.ecorrp = 0.0
    vpair = np.empty_like(rho)
    for iq in range(2):                                   # (370-382)
        v0 = f.v0prot if iq == 1 else f.v0neut
        if f.ipair == 6:
            vpair[iq] = v0 * chi[iq] * (1.0 - rt / f.rho0pr)
        else:
            vpair[iq] = v0 * chi[iq]
    mf.upot, mf.bmass, mf.divaq, mf.v_pair = upot, bmass, divaq, vpair
    mf.aq, mf.spot, mf.wlspot, mf.dbmass = aq, spot, wlspot, dbmass
    return mf, coulomb


def spectral_d1(n, d):
    """Dense first-derivative matrix with the k = 0 and n/2 bins zeroed (the
    first output of cderv00 / cderv02 as a matrix):
    D[j, l] = -(2 kf / n) sum_{k=1}^{n/2-1} k sin(2 pi k (j - l) / n)."""
    kf = 2.0 * np.pi / (n * d)
    j = np.arange(n)
    diff = j[:, None] - j[None, :]
    k = np.arange(1, n // 2)[:, None, None]
    return -(2.0 * kf / n) * np.sum(k * np.sin(2.0 * np.pi * k * diff / n), axis=0)


def hpsi01_matrix_form(grids, mf, iq, weight, weightuv, pinn):
    """hpsi01 (meanfield.py:41-159) in the form the single-precision
    tensor-core kernel evaluates, in FP64: along each axis d,
        out_d = L_d(D psi) + D(L_d psi - B D psi) + N_d,
    with D the dense derivative above, L_d the pointwise current /
    spin-orbit operator of axis d (the w of meanfield.py:77-84, 104-111,
    133-140) and N_d = (pi/d)^2 mean_line(B) (-1)^j sum_l (-1)^l psi_l / n
    the Nyquist bin cderv02 keeps (levels.py:314-315).  Equal to hpsi01 up
    to rounding; a single 2-spinor (2, nx, ny, nz)."""
    up, bm, aq, sp, wl, vp = (mf.upot[iq], mf.bmass[iq], mf.aq[iq], mf.spot[iq], mf.wlspot[iq], mf.v_pair[iq])
    p0, p1 = pinn[0], pinn[1]
    h = 0.5
    o0 = up * p0 + (sp[0] - 1j * sp[1]) * p1 + sp[2] * p0
    o1 = up * p1 + (sp[0] + 1j * sp[1]) * p0 - sp[2] * p1

    def L(axis, a0, a1):
        if axis == 0:
            return (-1j * h * (aq[0] - wl[1]) * a0 - h * wl[2] * a1,
                    -1j * h * (aq[0] + wl[1]) * a1 + h * wl[2] * a0)
        if axis == 1:
            return (-1j * h * (aq[1] + wl[0]) * a0 + 1j * h * wl[2] * a1,
                    -1j * h * (aq[1] - wl[0]) * a1 + 1j * h * wl[2] * a0)
        return (-1j * h * aq[2] * a0 + (h * wl[0] - 1j * h * wl[1]) * a1,
                -1j * h * aq[2] * a1 + (-h * wl[0] - 1j * h * wl[1]) * a0)

    for axis, d in enumerate((grids.dx, grids.dy, grids.dz)):
        n = pinn.shape[1 + axis]
        D = spectral_d1(n, d)
        e0, e1 = apply_along(D, p0, axis), apply_along(D, p1, axis)
        n0, n1 = L(axis, p0, p1)
        l0, l1 = L(axis, e0, e1)
        sign = (-1.0) ** np.arange(n)
        shp = [1, 1, 1]
        shp[axis] = n
        sign = sign.reshape(shp)
        bbar = np.mean(bm, axis=axis, keepdims=True)
        nq = (np.pi / d) ** 2 / n
        for c, (pc, ec, nc, lc) in enumerate(((p0, e0, n0, l0), (p1, e1, n1, l1))):
            alt = np.sum(sign * pc, axis=axis, keepdims=True)
            r = lc + apply_along(D, nc - bm * ec, axis) + nq * bbar * sign * alt
            if c == 0:
                o0 = o0 + r
            else:
                o1 = o1 + r
    pout_mf = np.stack([o0, o1])
    pout_del = pinn * vp
    return weight * pout_mf - weightuv * pout_del, pout_mf, pout_del
