"""Checkpoint files for the self-consistent loop.

The reference carries a ``trestart`` switch (params.py:74; static.py:1700-
1704 skips the first diagonalisation and starts at ``params.iteration + 1``)
but has no way to write or read a state.  This module adds one file format
and the two functions around it; ``hfb.static.prepare`` / ``statichf`` honour
``params.trestart`` as the reference's driver does.

File layout (all integers little-endian):

    bytes 0-7     magic  b"HFBRST01"
    bytes 8-15    uint64 length H of the header
    bytes 16..    H bytes of UTF-8 JSON:
                  {"format": "hfb-restart", "version": 1, "iteration": i,
                   "nneut": N, "nprot": Z, "npsi": [n0, n1],
                   "grid": {"nx", "ny", "nz", "dx", "dy", "dz"},
                   "arrays": {name: {"dtype", "shape", "offset"}}}
    arrays        raw C-order little-endian data, each starting at its
                  ``offset`` (absolute, a multiple of 64)

Arrays: the levels' ``psi`` (complex128 or complex64, as run), ``sp_energy``,
``sp_norm``, ``wocc``, ``wguv``, ``pairwg``, ``wstates``, ``deltaf`` and the
densities ``rho``, ``tau``, ``chi``, ``current``, ``sdens``, ``sodens``.
"""
import json
import struct

import numpy as np
import torch

MAGIC = b"HFBRST01"
LEVEL_ARRAYS = ("psi", "sp_energy", "sp_norm", "wocc", "wguv", "pairwg", "wstates", "deltaf")
DENSITY_ARRAYS = ("rho", "tau", "chi", "current", "sdens", "sodens")
_ALIGN = 64


def _grid_dict(grids):
    return dict(nx=int(grids.nx), ny=int(grids.ny), nz=int(grids.nz), dx=float(grids.dx), dy=float(grids.dy),
                dz=float(grids.dz))


def save_state(path, state):
    """Write the levels and densities of a state dict (from
    ``hfb.config.setup``) and the current iteration number to ``path``."""
    lv, dens, grids, params = state["levels"], state["densities"], state["grids"], state["params"]
    arrays = [(k, getattr(lv, k)) for k in LEVEL_ARRAYS] + [(k, getattr(dens, k)) for k in DENSITY_ARRAYS]
    host = [(k, t.detach().contiguous().cpu().numpy()) for k, t in arrays]
    meta = {}
    off = 0
    for k, a in host:
        meta[k] = dict(dtype=a.dtype.name, shape=list(a.shape), offset=off)
        off += -(-a.nbytes // _ALIGN) * _ALIGN
    hdr = dict(format="hfb-restart", version=1, iteration=int(params.iteration), nneut=int(lv.nneut),
               nprot=int(lv.nprot), npsi=[int(lv.npsi[0]), int(lv.npsi[1])], grid=_grid_dict(grids), arrays=meta)
    # array offsets are relative until the header length is known
    body = json.dumps(hdr).encode()
    start = -(-(16 + len(body) + 256) // _ALIGN) * _ALIGN
    for m in meta.values():
        m["offset"] += start
    body = json.dumps(hdr).encode()
    if 16 + len(body) > start:
        raise RuntimeError("restart header larger than reserved")
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(struct.pack("<Q", len(body)))
        f.write(body)
        for k, a in host:
            f.seek(meta[k]["offset"])
            f.write(np.ascontiguousarray(a).astype(a.dtype.newbyteorder("<"), copy=False).tobytes())


def read_header(path):
    """The JSON header of a restart file."""
    with open(path, "rb") as f:
        if f.read(8) != MAGIC:
            raise ValueError(f"{path}: not an hfb restart file")
        (h,) = struct.unpack("<Q", f.read(8))
        return json.loads(f.read(h).decode())


def load_state(path, state, densities=True):
    """Fill a state dict built by ``hfb.config.setup`` for the same nucleus,
    state counts and grid from ``path``; set ``params.iteration`` and
    ``params.trestart`` so that ``hfb.static.statichf`` continues from the
    saved iteration.  ``psi`` is converted to the state's precision.
    Returns the header."""
    hdr = read_header(path)
    lv, grids = state["levels"], state["grids"]
    if hdr.get("format") != "hfb-restart" or hdr.get("version") != 1:
        raise ValueError(f"{path}: unsupported restart format")
    if hdr["grid"] != _grid_dict(grids):
        raise ValueError(f"{path}: grid {hdr['grid']} differs from {_grid_dict(grids)}")
    if (hdr["nneut"], hdr["nprot"], list(hdr["npsi"])) != (lv.nneut, lv.nprot, [int(x) for x in lv.npsi]):
        raise ValueError(f"{path}: nucleus / state counts differ from the state's")
    names = list(LEVEL_ARRAYS) + (list(DENSITY_ARRAYS) if densities else [])
    with open(path, "rb") as f:
        for k in names:
            m = hdr["arrays"][k]
            dt = np.dtype(m["dtype"]).newbyteorder("<")
            n = int(np.prod(m["shape"])) if m["shape"] else 1
            f.seek(m["offset"])
            a = np.frombuffer(f.read(n * dt.itemsize), dtype=dt).reshape(m["shape"])
            dst = getattr(lv, k) if k in LEVEL_ARRAYS else getattr(state["densities"], k)
            if list(dst.shape) != list(m["shape"]):
                raise ValueError(f"{path}: {k} has shape {m['shape']}, the state {list(dst.shape)}")
            dst.copy_(torch.from_numpy(a.astype(a.dtype.newbyteorder("="))).to(dst.dtype))
    state["params"].iteration = int(hdr["iteration"])
    state["params"].trestart = True
    return hdr
