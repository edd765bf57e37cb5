"""Skyrme force and pairing parameters (mirror of forces.py:60-144).

The parameter table restates the reference's _forces.yml (SLy4).  ``h2ma``
is taken from the unscaled h2m (forces.py:141); init_static later rescales
h2m by (A-1)/A when zpe == 0 (static.py:87-88).
"""
from dataclasses import dataclass, field
import math

from ._lib import HfbForce

HBC = 197.328910
E2 = 1.4399784085965135

FORCE_TABLE = {
    "SLy4": dict(
        ex=1, zpe=0, h2m=(20.735530, 20.735530),
        t0=-2488.913, t1=486.818, t2=-546.395, t3=13777.0, t4=123.0,
        x0=0.834, x1=-0.344, x2=-1.0, x3=1.354, b4p=61.5, power=0.1666667,
        vdi=dict(v0prot=295.369, v0neut=286.669, rho0pr=0.0),
        dddi=dict(v0prot=-1.0, v0neut=-1.0, rho0pr=0.16),
    )
}

COUPLINGS = ("t0", "t1", "t2", "t3", "t4", "x0", "x1", "x2", "x3", "b4p", "power")


@dataclass
class Forces:
    name: str = "SLy4"
    ex: int = 1
    zpe: int = 0
    h2m: list = field(default_factory=lambda: [20.735530, 20.735530])
    t0: float = 0.0
    t1: float = 0.0
    t2: float = 0.0
    t3: float = 0.0
    t4: float = 0.0
    x0: float = 0.0
    x1: float = 0.0
    x2: float = 0.0
    x3: float = 0.0
    b4p: float = 0.0
    power: float = 0.0
    v0prot: float = 0.0
    v0neut: float = 0.0
    rho0pr: float = 0.16
    ipair: int = 0
    pair_reg: bool = False
    delta_fit: tuple = (-1.0, -1.0)
    pair_cutoff: tuple = (0.0, 0.0)
    state_cutoff: tuple = (0.0, 0.0)
    softcut_range: float = 0.1
    tbcs: bool = False
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

    def derive(self):
        """b- and C-coefficients (forces.py:95-122)."""
        self.b0 = self.t0 * (1.0 + 0.5 * self.x0)
        self.b0p = self.t0 * (0.5 + self.x0)
        self.b1 = (self.t1 * (1.0 + 0.5 * self.x1) + self.t2 * (1.0 + 0.5 * self.x2)) / 4.0
        self.b1p = (self.t1 * (0.5 + self.x1) - self.t2 * (0.5 + self.x2)) / 4.0
        self.b2 = (3.0 * self.t1 * (1.0 + 0.5 * self.x1) - self.t2 * (1.0 + 0.5 * self.x2)) / 8.0
        self.b2p = (3.0 * self.t1 * (0.5 + self.x1) + self.t2 * (0.5 + self.x2)) / 8.0
        self.b3 = self.t3 * (1.0 + 0.5 * self.x3) / 4.0
        self.b3p = self.t3 * (0.5 + self.x3) / 4.0
        self.b4 = self.t4 / 2.0
        self.slate = (3.0 / math.pi) ** (1.0 / 3.0) * E2
        self.Crho0 = 0.5 * self.b0 - 0.25 * self.b0p
        self.Crho1 = -0.25 * self.b0p
        self.Crho0D = self.b3 / 3.0 - self.b3p / 6.0
        self.Crho1D = -self.b3p / 6.0
        self.Cdrho0 = -0.5 * self.b2 + 0.25 * self.b2p
        self.Cdrho1 = 0.25 * self.b2p
        self.Ctau0 = self.b1 - 0.5 * self.b1p
        self.Ctau1 = -0.5 * self.b1p
        self.CdJ0 = -self.b4 - 0.5 * self.b4p
        self.CdJ1 = -0.5 * self.b4p
        return self

    def c_struct(self):
        """The hfb_force block passed to the library."""
        s = HfbForce()
        for k in ("b0", "b0p", "b1", "b1p", "b2", "b2p", "b3", "b3p", "b4", "b4p", "power", "slate", "h2ma",
                  "v0neut", "v0prot", "rho0pr", "Crho0", "Crho1", "Crho0D", "Crho1D", "Cdrho0", "Cdrho1", "Ctau0",
                  "Ctau1", "CdJ0", "CdJ1"):
            setattr(s, k, float(getattr(self, k)))
        s.h2m[0] = float(self.h2m[0])
        s.h2m[1] = float(self.h2m[1])
        s.ipair = int(self.ipair)
        s.ex = int(self.ex)
        s.zpe = int(self.zpe)
        return s


def init_forces(params=None, **kwargs):
    """forces.py:60-144.  ``overrides`` (dict) replaces t/x/W/power values
    (coupling sweeps); v0prot / v0neut / rho0pr override the table."""
    name = kwargs.get("name", "SLy4")
    if name not in FORCE_TABLE:
        raise KeyError(f"Force '{name}' not found in the force table.")
    src = dict(FORCE_TABLE[name])
    src.update(kwargs.get("overrides") or {})
    f = Forces(name=name, ex=src["ex"], zpe=src["zpe"], h2m=list(src["h2m"]),
               ipair=kwargs.get("ipair", 0), pair_reg=kwargs.get("pair_reg", False),
               delta_fit=tuple(kwargs.get("delta_fit", (-1.0, -1.0))),
               pair_cutoff=tuple(float(v) for v in kwargs.get("pair_cutoff", (0.0, 0.0))),
               state_cutoff=tuple(float(v) for v in kwargs.get("state_cutoff", (0.0, 0.0))),
               softcut_range=kwargs.get("softcut_range", 0.1), tbcs=bool(kwargs.get("tbcs", False)))
    for k in COUPLINGS:
        setattr(f, k, float(src[k]))
    f.derive()
    if f.ipair == 5:
        f.v0prot, f.v0neut, f.rho0pr = src["vdi"]["v0prot"], src["vdi"]["v0neut"], src["vdi"]["rho0pr"]
    if f.ipair == 6:
        f.v0prot, f.v0neut, f.rho0pr = src["dddi"]["v0prot"], src["dddi"]["v0neut"], src["dddi"]["rho0pr"]
    for k in ("v0prot", "v0neut", "rho0pr"):
        if k in kwargs:
            setattr(f, k, float(kwargs[k]))
    f.h2ma = 0.5 * (f.h2m[0] + f.h2m[1])
    f.nucleon_mass = HBC ** 2 / (2.0 * f.h2ma)
    return f
