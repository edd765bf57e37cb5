"""Constants, Skyrme force, grid and level set-up (oracle; test infrastructure).

Follows reference params.py:48-95, forces.py:60-144, grids.py:36-138,
levels.py:37-130 and static.py:53-90.
"""
from dataclasses import dataclass, field
import numpy as np

# params.py:53-54
HBC = 197.328910
E2 = 1.4399784085965135

# _forces.yml:1-25 (SLy4, Chabanat et al. 1998), the only set the reference ships.
FORCE_TABLE = {
    "SLy4": dict(
        ex=1, zpe=0, h2m=(20.735530, 20.735530),
        t0=-2488.913, t1=486.818, t2=-546.395, t3=13777.0, t4=123.0,
        x0=0.834, x1=-0.344, x2=-1.0, x3=1.354, b4p=61.5, power=0.1666667,
        vdi=dict(v0prot=295.369, v0neut=286.669, rho0pr=0.0),
        dddi=dict(v0prot=-1.0, v0neut=-1.0, rho0pr=0.16),
    )
}


@dataclass
class Forces:
    name: str
    ex: int
    zpe: int
    h2m: np.ndarray
    t0: float
    t1: float
    t2: float
    t3: float
    t4: float
    x0: float
    x1: float
    x2: float
    x3: float
    b4p: float
    power: float
    v0prot: float
    v0neut: float
    rho0pr: float
    ipair: int
    pair_reg: bool
    delta_fit: np.ndarray
    pair_cutoff: np.ndarray
    state_cutoff: np.ndarray
    softcut_range: float
    tbcs: bool
    h2ma: float = 0.0
    nucleon_mass: float = 0.0
    b0: float = 0.0
    b0p: float = 0.0
    b1: float = 0.0
    b1p: float = 0.0
    b2: float = 0.0
    b2p: float = 0.0
    b3: float = 0.0
    b3p: float = 0.0
    b4: float = 0.0
    slate: float = 0.0
    Crho0: float = 0.0
    Crho1: float = 0.0
    Crho0D: float = 0.0
    Crho1D: float = 0.0
    Cdrho0: float = 0.0
    Cdrho1: float = 0.0
    Ctau0: float = 0.0
    Ctau1: float = 0.0
    CdJ0: float = 0.0
    CdJ1: float = 0.0


def derive_coefficients(f):
    """b- and C-coefficients from t/x parameters (forces.py:95-122)."""
    f.b0 = f.t0 * (1.0 + 0.5 * f.x0)
    f.b0p = f.t0 * (0.5 + f.x0)
    f.b1 = (f.t1 * (1.0 + 0.5 * f.x1) + f.t2 * (1.0 + 0.5 * f.x2)) / 4.0
    f.b1p = (f.t1 * (0.5 + f.x1) - f.t2 * (0.5 + f.x2)) / 4.0
    f.b2 = (3.0 * f.t1 * (1.0 + 0.5 * f.x1) - f.t2 * (1.0 + 0.5 * f.x2)) / 8.0
    f.b2p = (3.0 * f.t1 * (0.5 + f.x1) + f.t2 * (0.5 + f.x2)) / 8.0
    f.b3 = f.t3 * (1.0 + 0.5 * f.x3) / 4.0
    f.b3p = f.t3 * (0.5 + f.x3) / 4.0
    f.b4 = f.t4 / 2.0
    f.slate = (3.0 / np.pi) ** (1.0 / 3.0) * E2
    f.Crho0 = 0.5 * f.b0 - 0.25 * f.b0p
    f.Crho1 = -0.25 * f.b0p
    f.Crho0D = f.b3 / 3.0 - f.b3p / 6.0
    f.Crho1D = -f.b3p / 6.0
    f.Cdrho0 = -0.5 * f.b2 + 0.25 * f.b2p
    f.Cdrho1 = 0.25 * f.b2p
    f.Ctau0 = f.b1 - 0.5 * f.b1p
    f.Ctau1 = -0.5 * f.b1p
    f.CdJ0 = -f.b4 - 0.5 * f.b4p
    f.CdJ1 = -0.5 * f.b4p
    return f


def init_forces(name="SLy4", ipair=0, tbcs=False, pair_reg=False, delta_fit=(-1.0, -1.0),
                pair_cutoff=(0.0, 0.0), state_cutoff=(0.0, 0.0), softcut_range=0.1,
                overrides=None, **pairing):
    """forces.py:60-144.  ``overrides`` replaces t/x/W parameters (used by the
    coupling-perturbation tests); ``pairing`` may hold v0prot/v0neut/rho0pr."""
    src = dict(FORCE_TABLE[name])
    if overrides:
        src.update(overrides)
    f = Forces(name=name, ex=src["ex"], zpe=src["zpe"], h2m=np.array(src["h2m"], dtype=np.float64),
               t0=src["t0"], t1=src["t1"], t2=src["t2"], t3=src["t3"], t4=src["t4"],
               x0=src["x0"], x1=src["x1"], x2=src["x2"], x3=src["x3"], b4p=src["b4p"],
               power=src["power"], v0prot=0.0, v0neut=0.0, rho0pr=0.16, ipair=ipair,
               pair_reg=pair_reg, delta_fit=np.array(delta_fit, dtype=np.float64),
               pair_cutoff=np.array(pair_cutoff, dtype=np.float64),
               state_cutoff=np.array(state_cutoff, dtype=np.float64),
               softcut_range=softcut_range, tbcs=tbcs)
    derive_coefficients(f)
    if ipair == 5:
        f.v0prot, f.v0neut, f.rho0pr = src["vdi"]["v0prot"], src["vdi"]["v0neut"], src["vdi"]["rho0pr"]
    if ipair == 6:
        f.v0prot, f.v0neut, f.rho0pr = src["dddi"]["v0prot"], src["dddi"]["v0neut"], src["dddi"]["rho0pr"]
    for k in ("v0prot", "v0neut", "rho0pr"):
        if k in pairing:
            setattr(f, k, pairing[k])
    # h2ma is taken from the unscaled h2m (forces.py:141) before init_static rescales h2m.
    f.h2ma = float(0.5 * np.sum(f.h2m))
    f.nucleon_mass = HBC ** 2 / (2.0 * f.h2ma)
    return f


def sder(n, d):
    """Dense spectral first-derivative matrix (grids.py:36-46)."""
    icn = (n + 1) // 2
    afac = np.pi / icn
    idx = np.arange(1, n + 1)
    diff = idx[None, :] - idx[:, None]
    j = np.arange(1, icn)[:, None, None]
    s = np.sum(-j * np.sin(j * afac * diff), axis=0)
    return -afac * (s - 0.5 * icn * np.sin(icn * afac * diff)) / (icn * d)


def sder2(n, d):
    """Dense spectral second-derivative matrix (grids.py:51-61)."""
    icn = (n + 1) // 2
    afac = np.pi / icn
    idx = np.arange(1, n + 1)
    diff = idx[None, :] - idx[:, None]
    j = np.arange(1, icn)[:, None, None]
    s = np.sum(j ** 2 * np.cos(j * afac * diff), axis=0)
    return -(afac * afac) * (s + 0.5 * icn ** 2 * np.cos(icn * afac * diff)) / (icn * d * d)


@dataclass
class Grids:
    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float
    periodic: bool
    wxyz: float
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    der1: list = field(default_factory=list)   # [der1x, der1y, der1z]
    der2: list = field(default_factory=list)

    @property
    def n(self):
        return (self.nx, self.ny, self.nz)

    @property
    def d(self):
        return (self.dx, self.dy, self.dz)


def init_grids(nx=48, ny=48, nz=48, dx=0.8, dy=0.8, dz=0.8, periodic=False):
    """grids.py:66-138 (no Bloch phases / TABC, which the reference leaves unimplemented)."""
    for v in (nx, ny, nz):
        if v % 2 != 0:
            raise ValueError("grids: nx, ny, and nz must be even.")
    if dx * dy * dz <= 0.0:
        if dx <= 0.0:
            raise ValueError("grid spacing given as 0.")
        dy = dz = dx

    def centred(n, d):
        return (np.arange(n, dtype=np.float64) - (n - 1) / 2.0) * d

    g = Grids(nx=nx, ny=ny, nz=nz, dx=dx, dy=dy, dz=dz, periodic=periodic, wxyz=dx * dy * dz,
              x=centred(nx, dx), y=centred(ny, dy), z=centred(nz, dz))
    g.der1 = [sder(nx, dx), sder(ny, dy), sder(nz, dz)]
    g.der2 = [sder2(nx, dx), sder2(ny, dy), sder2(nz, dz)]
    return g


def apply_along(mat, f, axis):
    """out[..i..] = sum_j mat[i, j] f[..j..] along ``axis`` of a 3-D field
    (the einsum patterns 'ij,jkl->ikl', 'jl,ilk->ijk', 'kl,ijl->ijk' of
    meanfield.py:197-199)."""
    return np.moveaxis(np.tensordot(mat, f, axes=([1], [axis])), 0, axis)


@dataclass
class Levels:
    nneut: int
    nprot: int
    npsi: tuple
    nstmax: int
    charge_number: int
    mass_number: int
    isospin: np.ndarray
    psi: np.ndarray
    hampsi: np.ndarray
    lagrange: np.ndarray
    hmfpsi: np.ndarray
    delpsi: np.ndarray
    sp_energy: np.ndarray
    sp_efluct1: np.ndarray
    sp_efluct2: np.ndarray
    sp_kinetic: np.ndarray
    sp_norm: np.ndarray
    sp_orbital: np.ndarray
    sp_spin: np.ndarray
    sp_parity: np.ndarray
    wocc: np.ndarray
    wguv: np.ndarray
    pairwg: np.ndarray
    wstates: np.ndarray
    deltaf: np.ndarray

    def block(self, iq):
        """Slice of the states of isospin ``iq`` (neutrons first, levels.py:54)."""
        s = 0 if iq == 0 else self.npsi[0]
        return slice(s, s + self.npsi[iq])


def init_levels(grids, nneut, nprot, npsi=None):
    """levels.py:37-130."""
    if npsi is None:
        npsi = (max(126, nneut + int(1.65 * nneut ** 0.666667)),
                max(82, nprot + int(1.65 * nprot ** 0.666667)))
    npsi = (int(npsi[0]), int(npsi[1]))
    nst = npsi[0] + npsi[1]
    shp = (nst, 2, grids.nx, grids.ny, grids.nz)
    z = lambda: np.zeros(shp, dtype=np.complex128)
    iso = np.zeros(nst, dtype=np.int32)
    iso[npsi[0]:] = 1
    wocc = np.zeros(nst)
    wocc[:nneut] = 1.0
    wocc[npsi[0]:npsi[0] + nprot] = 1.0
    return Levels(nneut=nneut, nprot=nprot, npsi=npsi, nstmax=nst, charge_number=nprot,
                  mass_number=nneut + nprot, isospin=iso, psi=z(), hampsi=z(), lagrange=z(),
                  hmfpsi=z(), delpsi=z(), sp_energy=np.zeros(nst), sp_efluct1=np.zeros(nst),
                  sp_efluct2=np.zeros(nst), sp_kinetic=np.zeros(nst), sp_norm=np.zeros(nst),
                  sp_orbital=np.zeros((nst, 3)), sp_spin=np.zeros((nst, 3)), sp_parity=np.zeros(nst),
                  wocc=wocc, wguv=np.zeros(nst), pairwg=np.ones(nst), wstates=np.ones(nst),
                  deltaf=np.zeros(nst))
