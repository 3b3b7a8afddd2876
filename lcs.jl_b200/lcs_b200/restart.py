"""Restart files in the reference's HDF5 layout (src/LCSIO/save.jl:40-167,
load.jl:23-118), through the library's own reader and writer
(csrc/lcs_h5.cpp): no HDF5 library is needed.

    save(engine, "restart.h5.100")      # /flow/{U,V,W,P}, /particles/<i>/...
    load(engine, "restart.h5.100")      # same dims and particle counts
    load_coarse(engine, "restart.h5.0") # the `upsample` init from half dims
    dataset(path, "flow/U")             # any dataset of the supported subset
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from .engine import LCSError


def _err(lib, rc):
    if rc != 0:
        raise LCSError(rc, lib.lcs_io_last_error().decode())


def save(engine, path: str):
    _err(engine.lib, engine.lib.lcs_restart_save(engine.handle, path.encode()))


def load(engine, path: str):
    _err(engine.lib, engine.lib.lcs_restart_load(engine.handle, path.encode()))


def load_coarse(engine, path: str):
    _err(engine.lib, engine.lib.lcs_restart_load_coarse(engine.handle, path.encode()))


def save_state(lib, path: str, step: int, t: float, dt: float):
    _err(lib, lib.lcs_stat_state_save(path.encode(), step, t, dt))


def save_stat(lib, path: str, step: int, t: float, dt: float, flow=None, nvalid=None, particles=None, log=None):
    """`LCSIO.savestat` of one step (lcs_stat_save): `flow` a FlowStat (or its
    dict), `nvalid` the species' particle counts, `particles` a sequence of
    ParticleStats, `log` a Log; each may be None."""
    fs = None
    if flow is not None:
        fs = flow if isinstance(flow, _abi.FlowStat) else _abi.FlowStat(**flow)
    ns = len(particles) if particles is not None else (len(nvalid) if nvalid is not None else 0)
    nv = (C.c_int64 * max(ns, 1))(*nvalid) if nvalid is not None else None
    ps = (_abi.ParticleStats * max(ns, 1))(*particles) if particles is not None else None
    _err(lib, lib.lcs_stat_save(path.encode(), step, t, dt, C.byref(fs) if fs is not None else None, ns,
                                nv, ps, C.byref(log) if log is not None else None))


def load_state(lib, path: str, step: int):
    t, dt = C.c_double(), C.c_double()
    _err(lib, lib.lcs_stat_state_load(path.encode(), step, C.byref(t), C.byref(dt)))
    return t.value, dt.value


def dataset(lib, path: str, name: str) -> np.ndarray:
    """A dataset as a numpy array of its HDF5 dims (float64 or int64)."""
    rank, dims, kind = C.c_int32(), (C.c_int64 * 8)(), C.create_string_buffer(1)
    _err(lib, lib.lcs_h5_dataset(path.encode(), name.encode(), C.byref(rank), dims, kind, None, 0))
    shape = tuple(dims[q] for q in range(rank.value))
    out = np.empty(shape, dtype=np.float64 if kind.raw == b"f" else np.int64)
    _err(lib, lib.lcs_h5_dataset(path.encode(), name.encode(), C.byref(rank), dims, kind,
                                 out.ctypes.data_as(C.c_void_p), out.nbytes))
    return out


def listing(lib, path: str, group: str = "/") -> list:
    buf = C.create_string_buffer(1 << 16)
    _err(lib, lib.lcs_h5_list(path.encode(), group.encode(), buf, len(buf)))
    return [n for n in buf.value.decode().split("\n") if n]
