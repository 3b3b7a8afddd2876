"""The batching and serving forms of include/lcs_b200.h (no reference
counterpart), with numpy in and out.

Batch: an ensemble of independent runs (uneven sizes, particle counts and
parameters) stepped together; members are Engine views for uploads and
downloads.  Server: continuous batching of simulation requests admitted by
device-memory footprint, with p50/p99 latency.

Both take the library to drive (`lib`): the CUDA library by default, or any
library with the same ABI (the tests also run them over the CPU oracle).
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from .engine import Engine, LCSError, _c64, _dptr


def _serve_check(lib, rc: int):
    if rc != 0:
        raise LCSError(rc, lib.lcs_serve_last_error().decode())


class Batch:
    """`lcs_batch_*`: members advance together, each exactly as it would alone."""

    def __init__(self, configs, lib=None):
        self.lib = lib if lib is not None else _abi.load_library()
        self.configs = list(configs)
        arr = (_abi.Config * len(self.configs))(*self.configs)
        b = C.c_void_p()
        _serve_check(self.lib, self.lib.lcs_batch_create(arr, len(self.configs), C.byref(b)))
        self.handle = b
        self.members = []
        for i, cfg in enumerate(self.configs):
            h = C.c_void_p()
            _serve_check(self.lib, self.lib.lcs_batch_member(self.handle, i, C.byref(h)))
            self.members.append(Engine.borrow(self.lib, cfg, h))

    def __len__(self):
        return len(self.members)

    def tuning(self, i: int) -> dict:
        """The launch shapes the batch's autotuner chose for member i."""
        rows, zc = C.c_int32(), C.c_int32()
        share, ms = C.c_double(), C.c_double()
        _serve_check(self.lib, self.lib.lcs_batch_tuning(self.handle, i, C.byref(rows), C.byref(zc), C.byref(share),
                                                         C.byref(ms)))
        return {"rw_rows": rows.value, "zchunk": zc.value, "share": share.value, "probe_ms": ms.value}

    def step(self, nsteps: int) -> list:
        """nsteps of every member; returns logs[member][step] as dicts."""
        m = len(self.members)
        logs = (_abi.Log * max(1, m * nsteps))()
        _serve_check(self.lib, self.lib.lcs_batch_step(self.handle, nsteps, logs))
        return [[logs[i * nsteps + q].as_dict() for q in range(nsteps)] for i in range(m)]

    def close(self):
        if getattr(self, "handle", None):
            for e in self.members:
                e.close()
            self.lib.lcs_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """`lcs_server_*`: a request loop with continuous batching."""

    def __init__(self, device: int = 0, max_active: int = 8, steps_per_slice: int = 4,
                 hbm_budget_bytes: int = 150 * 10 ** 9, lib=None):
        self.lib = lib if lib is not None else _abi.load_library()
        sc = _abi.ServerConfig(device=device, max_active=max_active, steps_per_slice=steps_per_slice,
                               hbm_budget_bytes=int(hbm_budget_bytes))
        s = C.c_void_p()
        _serve_check(self.lib, self.lib.lcs_server_create(C.byref(sc), C.byref(s)))
        self.handle = s
        self._cfgs = {}

    def submit(self, cfg: _abi.Config, U, V, W, P, species=(), nsteps: int = 1, interp_velocity: bool = True) -> int:
        """species: per species a dict with diam, x, y, z, u, v, w (and optional ids)."""
        req = _abi.Request()
        req.config = cfg
        keep = [_c64(a).ravel() for a in (U, V, W, P)]
        req.U, req.V, req.W, req.P = (_dptr(a) for a in keep)
        for s, sp in enumerate(species):
            arrs = {k: _c64(sp[k]) for k in ("diam", "x", "y", "z", "u", "v", "w")}
            keep.extend(arrs.values())
            st = req.species[s]
            for k, a in arrs.items():
                setattr(st, k, _dptr(a))
            if sp.get("ids") is not None:
                ids = np.ascontiguousarray(sp["ids"], dtype=np.int64)
                keep.append(ids)
                st.ids = ids.ctypes.data_as(C.POINTER(C.c_int64))
        req.interp_velocity = int(interp_velocity)
        req.nsteps = int(nsteps)
        t = C.c_int64()
        _serve_check(self.lib, self.lib.lcs_server_submit(self.handle, C.byref(req), C.byref(t)))
        self._cfgs[t.value] = cfg
        return t.value

    def poll(self, ticket: int):
        st, done = C.c_int32(), C.c_int64()
        _serve_check(self.lib, self.lib.lcs_server_poll(self.handle, ticket, C.byref(st), C.byref(done)))
        return st.value, done.value

    def result(self, ticket: int) -> dict:
        cfg = self._cfgs[ticket]
        n3 = int(cfg.dims[0]) * int(cfg.dims[1]) * int(cfg.dims[2])
        shape = (int(cfg.dims[2]), int(cfg.dims[1]), int(cfg.dims[0]))
        flow = [np.empty(shape) for _ in range(4)]
        ns = int(cfg.n_species) if cfg.mode == _abi.MODE_FLOW_PARTICLE else 0
        outs = (_abi.SpeciesOut * max(1, ns))()
        parts = []
        for s in range(ns):
            n = int(cfg.species[s].nvalid)
            d = {k: np.empty(n) for k in ("x", "y", "z", "u", "v", "w")}
            for k, a in d.items():
                setattr(outs[s], k, _dptr(a))
            parts.append(d)
        log = _abi.Log()
        lat = C.c_double()
        _serve_check(self.lib, self.lib.lcs_server_result(self.handle, ticket, *[_dptr(a) for a in flow], outs,
                                                          C.byref(log), C.byref(lat)))
        assert flow[0].size == n3
        return {"flow": flow, "particles": parts, "log": log.as_dict(), "latency_s": lat.value}

    def release(self, ticket: int):
        _serve_check(self.lib, self.lib.lcs_server_release(self.handle, ticket))
        self._cfgs.pop(ticket, None)

    def stats(self) -> dict:
        st = _abi.ServerStats()
        _serve_check(self.lib, self.lib.lcs_server_stats_get(self.handle, C.byref(st)))
        return st.as_dict()

    def drain(self, timeout_s: float = 600.0):
        _serve_check(self.lib, self.lib.lcs_server_drain(self.handle, timeout_s))

    def close(self):
        if getattr(self, "handle", None):
            self.lib.lcs_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
