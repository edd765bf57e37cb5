"""Run parameters (mirror of params.py:48-95 of jax-hfbfft)."""
from dataclasses import dataclass

import math


@dataclass
class Params:
    pi: float = math.pi
    hbc: float = 197.328910
    e2: float = 1.4399784085965135
    r0: float = 1.2
    tcoul: bool = True
    tstatic: bool = True
    tdynamic: bool = False
    tfft: bool = True
    trestart: bool = False
    mprint: int = 10
    mplot: int = 0
    mrest: int = 0
    iteration: int = 0
    time: float = 0.0
    nof: int = 0
    tabc_nprocs: int = 1
    tabc_myid: int = 0
    wffile: str = "none"


def init_params(**kwargs):
    """params.py:48-95: ``imode`` selects static (1) or dynamic (0)."""
    imode = kwargs.pop("imode", 1)
    known = {f for f in Params.__dataclass_fields__}
    p = Params(**{k: v for k, v in kwargs.items() if k in known})
    p.tstatic = imode == 1
    p.tdynamic = imode == 0
    return p
