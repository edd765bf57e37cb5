"""Single-particle states and spectral derivatives (mirror of levels.py).

``psi[nst, 2, nx, ny, nz]`` is complex128 (FP64 path) or complex64 (FP32
path), neutrons first (levels.py:54).
"""
from dataclasses import dataclass
import ctypes as C

import torch

from . import _lib
from ._lib import call, ptr, stream_ptr, prec_of


@dataclass
class Levels:
    nstmax: int
    nneut: int
    nprot: int
    npsi: tuple
    charge_number: int
    mass_number: int
    psi: torch.Tensor
    hampsi: torch.Tensor
    lagrange: torch.Tensor
    hmfpsi: torch.Tensor
    delpsi: torch.Tensor
    psi_spare: torch.Tensor
    isospin: torch.Tensor
    sp_energy: torch.Tensor
    sp_efluct1: torch.Tensor
    sp_efluct2: torch.Tensor
    sp_kinetic: torch.Tensor
    sp_norm: torch.Tensor
    sp_orbital: torch.Tensor
    sp_spin: torch.Tensor
    sp_parity: torch.Tensor
    wocc: torch.Tensor
    wguv: torch.Tensor
    pairwg: torch.Tensor
    wstates: torch.Tensor
    deltaf: torch.Tensor

    @property
    def npmin(self):
        return (0, self.npsi[0])

    @property
    def dtype(self):
        return self.psi.dtype

    def to_precision(self, dtype):
        """Convert the state arrays to complex128 / complex64 in place."""
        for k in ("psi", "hampsi", "lagrange", "hmfpsi", "delpsi", "psi_spare"):
            t = getattr(self, k)
            if t is not None and t.dtype != dtype:
                setattr(self, k, t.to(dtype))
        return self


def init_levels(grids, nneut=82, nprot=50, npsi=None, dtype=torch.complex128, store_delpsi=False):
    """levels.py:37-130.  ``store_delpsi`` keeps v_pair*psi as an array; the
    iteration itself recomputes it inside the Gram contraction."""
    if npsi is None:
        npsi = (max(126, nneut + int(1.65 * nneut ** 0.666667)), max(82, nprot + int(1.65 * nprot ** 0.666667)))
    npsi = (int(npsi[0]), int(npsi[1]))
    nst = npsi[0] + npsi[1]
    dev = torch.device("cuda")
    shp = (nst, 2, grids.nx, grids.ny, grids.nz)

    def z():
        return torch.zeros(shp, dtype=dtype, device=dev)

    def r(v=0.0):
        return torch.full((nst,), v, dtype=torch.float64, device=dev)

    iso = torch.zeros(nst, dtype=torch.int32, device=dev)
    iso[npsi[0]:] = 1
    wocc = r()
    wocc[:nneut] = 1.0
    wocc[npsi[0]:npsi[0] + nprot] = 1.0
    lv = Levels(nstmax=nst, nneut=nneut, nprot=nprot, npsi=npsi, charge_number=nprot, mass_number=nneut + nprot,
                  psi=z(), hampsi=z(), lagrange=z(), hmfpsi=z(), delpsi=z() if store_delpsi else None,
                  psi_spare=z(), isospin=iso, sp_energy=r(), sp_efluct1=r(), sp_efluct2=r(), sp_kinetic=r(),
                  sp_norm=r(), sp_orbital=torch.zeros((nst, 3), dtype=torch.float64, device=dev),
                  sp_spin=torch.zeros((nst, 3), dtype=torch.float64, device=dev), sp_parity=r(), wocc=wocc,
                  wguv=r(), pairwg=r(1.0), wstates=r(1.0), deltaf=r())
    lv._ctx = grids.ctx
    return lv


# --------------------------------------------------------- derivatives ----
def _cderv(grids, kind, axis, psin, bfield=None):
    x = psin.contiguous()
    nsp = x.numel() // (2 * grids.n3)
    d1 = torch.empty_like(x)
    d2 = torch.empty_like(x) if kind > 0 else None
    bf = bfield.contiguous().to(torch.float64) if bfield is not None else None
    call("hfb_cderv", grids.ctx.handle, prec_of(x), kind, axis, nsp, ptr(x), ptr(bf), ptr(d1), ptr(d2),
         stream_ptr())
    return d1 if kind == 0 else (d1, d2)


def _grid_of(d):
    g = _CURRENT_GRID.get("g")
    if g is None:
        raise RuntimeError("call hfb.levels.use_grid(grids) before the cderv functions")
    return g


_CURRENT_GRID = {}


def use_grid(grids):
    """The reference's cderv functions take only the spacing; the grid (and
    its device context) used by them is registered here."""
    _CURRENT_GRID["g"] = grids


def cdervx00(d, psin):
    return _cderv(_grid_of(d), 0, 0, psin)


def cdervy00(d, psin):
    return _cderv(_grid_of(d), 0, 1, psin)


def cdervz00(d, psin):
    return _cderv(_grid_of(d), 0, 2, psin)


def cdervx01(d, psin):
    return _cderv(_grid_of(d), 1, 0, psin)


def cdervy01(d, psin):
    return _cderv(_grid_of(d), 1, 1, psin)


def cdervz01(d, psin):
    return _cderv(_grid_of(d), 1, 2, psin)


def cdervx02(d, psin, pos_func):
    return _cderv(_grid_of(d), 2, 0, psin, pos_func)


def cdervy02(d, psin, pos_func):
    return _cderv(_grid_of(d), 2, 1, psin, pos_func)


def cdervz02(d, psin, pos_func):
    return _cderv(_grid_of(d), 2, 2, psin, pos_func)


def laplace(nst, iq, grids, forces, levels, wg, wguv, psin, v_pairmax, e0inv):
    """(E0 + T)^-1 preconditioner (levels.py:398-437) on one spinor or a
    batch of spinors; ``wg`` / ``wguv`` are scalars or per-spinor tensors."""
    x = psin.contiguous()
    nsp = x.numel() // (2 * grids.n3)
    dev = x.device
    wg_t = torch.as_tensor(wg, dtype=torch.float64, device=dev).reshape(-1).expand(nsp).contiguous()
    wu_t = torch.as_tensor(wguv, dtype=torch.float64, device=dev).reshape(-1).expand(nsp).contiguous()
    out = torch.empty_like(x)
    call("hfb_laplace", grids.ctx.handle, prec_of(x), nsp, ptr(x), ptr(wg_t), ptr(wu_t), float(v_pairmax),
         float(e0inv), float(forces.h2ma), ptr(out), stream_ptr())
    return out
