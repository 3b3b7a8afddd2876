"""Engine: one time-step handle of the C ABI, with numpy in and out.

Field arrays are numpy ``float64`` arrays indexed ``[k, j, i]`` (C order), so
x is the fastest axis exactly as in the reference's column-major Julia arrays.
The methods mirror the reference's functions one to one; the docstrings name
the Julia function each replaces.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi


class LCSError(RuntimeError):
    """A non-zero status of the C ABI (the reference raises ArgumentError)."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{_abi.ERROR_NAMES.get(code, code)}: {message}")
        self.code = code


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _c64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


class Engine:
    """A handle of ``liblcs_b200.so`` (the CUDA implementation)."""

    @staticmethod
    def _load():
        return _abi.load_library()

    def __init__(self, cfg: _abi.Config):
        self.lib = self._load()
        self.cfg = cfg
        self.n = tuple(int(d) for d in cfg.dims)
        self.h = int(cfg.halo_size)
        h = C.c_void_p()
        rc = self.lib.lcs_create(C.byref(cfg), C.byref(h))
        if rc != 0:
            raise LCSError(rc, self.lib.lcs_last_error(None).decode())
        self.handle = h

    @classmethod
    def borrow(cls, lib, cfg: _abi.Config, handle) -> "Engine":
        """A view of a handle owned elsewhere (a batch member): every method
        works, and close() leaves the handle to its owner."""
        e = cls.__new__(cls)
        e.lib, e.cfg = lib, cfg
        e.n = tuple(int(d) for d in cfg.dims)
        e.h = int(cfg.halo_size)
        e.handle = handle
        e._borrowed = True
        return e

    # -- lifetime ----------------------------------------------------------
    def close(self):
        if getattr(self, "handle", None):
            if not getattr(self, "_borrowed", False):
                self.lib.lcs_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int):
        if rc != 0:
            raise LCSError(rc, self.lib.lcs_last_error(self.handle).decode())

    @property
    def interior_shape(self):
        nx, ny, nz = self.n
        return (nz, ny, nx)

    @property
    def haloed_shape(self):
        nx, ny, nz = self.n
        h = self.h
        return (nz + 2 * h, ny + 2 * h, nx + 2 * h)

    # -- state transfer ----------------------------------------------------
    def upload_flow(self, U, V, W, P):
        """`Flows.init!` target: interior U, V, W, P (src/flows/inits)."""
        arrs = [_c64(a).reshape(self.interior_shape) for a in (U, V, W, P)]
        self._check(self.lib.lcs_upload_flow(self.handle, *[_dptr(a) for a in arrs]))

    def upload_flow_coarse(self, U, V, W, P):
        """The `upsample` init (src/LCSIO/upsample.jl:1-91): coarse (n/2)^3
        interior arrays [k, j, i], upsampled 2x on the device."""
        arrs = [_c64(a) for a in (U, V, W, P)]
        self._check(self.lib.lcs_upload_flow_coarse(self.handle, *[_dptr(a) for a in arrs]))

    def download_flow(self):
        out = [np.empty(self.interior_shape) for _ in range(4)]
        self._check(self.lib.lcs_download_flow(self.handle, *[_dptr(a) for a in out]))
        return out

    def field_set(self, field: int, data, haloed: bool = False):
        shape = self.haloed_shape if (haloed and field <= _abi.FIELD_P) else self.interior_shape
        a = _c64(data).reshape(shape)
        self._check(self.lib.lcs_field_set(self.handle, field, _dptr(a), int(haloed)))

    def field_get(self, field: int, haloed: bool = False) -> np.ndarray:
        shape = self.haloed_shape if (haloed and field <= _abi.FIELD_P) else self.interior_shape
        out = np.empty(shape)
        self._check(self.lib.lcs_field_get(self.handle, field, _dptr(out), int(haloed)))
        return out

    def upload_particles(self, species: int, diam, x, y, z, u, v, w, ids=None):
        arrs = [_c64(a) for a in (diam, x, y, z, u, v, w)]
        n = arrs[1].size
        idp = None
        if ids is not None:
            ids = np.ascontiguousarray(ids, dtype=np.int64)
            idp = ids.ctypes.data_as(C.POINTER(C.c_int64))
        self._check(self.lib.lcs_upload_particles(self.handle, species, n, idp, *[_dptr(a) for a in arrs]))

    def download_particles(self, species: int) -> dict:
        n = int(self.cfg.species[species].nvalid)
        ids = np.empty(n, dtype=np.int64)
        out = [np.empty(n) for _ in range(7)]
        self._check(
            self.lib.lcs_download_particles(
                self.handle, species, ids.ctypes.data_as(C.POINTER(C.c_int64)), *[_dptr(a) for a in out]
            )
        )
        return dict(zip(["diam", "x", "y", "z", "u", "v", "w"], out), ids=ids)

    def prop_set(self, species: int, prop: int, data):
        a = _c64(data)
        self._check(self.lib.lcs_prop_set(self.handle, species, prop, _dptr(a)))

    def prop_get(self, species: int, prop: int) -> np.ndarray:
        out = np.empty(int(self.cfg.species[species].nvalid))
        self._check(self.lib.lcs_prop_get(self.handle, species, prop, _dptr(out)))
        return out

    def set_state(self, step: int, t: float):
        self._check(self.lib.lcs_set_state(self.handle, step, t))

    def get_state(self):
        step = C.c_int64()
        t = C.c_double()
        self._check(self.lib.lcs_get_state(self.handle, C.byref(step), C.byref(t)))
        return step.value, t.value

    # -- the per-step calls ---------------------------------------------------
    def timestep(self) -> float:
        """`LCS.timestep` (src/timestep.jl:14-27)."""
        dt = C.c_double()
        self._check(self.lib.lcs_timestep(self.handle, C.byref(dt)))
        return dt.value

    def evolve(self, dt: float) -> dict:
        """`LCS.evolve!` (src/evolve.jl:63-146) with state.dt = dt."""
        log = _abi.Log()
        self._check(self.lib.lcs_evolve(self.handle, dt, C.byref(log)))
        return log.as_dict()

    def step(self, nsteps: int, logs: bool = True):
        """nsteps x (timestep! + evolve!) with no host round trip in between."""
        arr = (_abi.Log * max(1, nsteps))() if logs else None
        self._check(self.lib.lcs_step(self.handle, nsteps, arr if logs else None))
        return [arr[q].as_dict() for q in range(nsteps)] if logs else None

    def particles_makeindex(self, species: int, stage: int, grid_ratio: int):
        """`Particles.makeindex!` (src/particles/makeindex.jl:29-67): sorts the species by cell hash."""
        self._check(self.lib.lcs_particles_makeindex(self.handle, species, stage, grid_ratio))

    def set_particle_sort(self, interval: int, grid_ratio: int = 4):
        """Keep particles in cell order: makeindex! of every species after every
        `interval`-th step of `step` (0 turns it off); ids follow the order."""
        self._check(self.lib.lcs_set_particle_sort(self.handle, interval, grid_ratio))

    def particles_cellindex(self, species: int, grid_ratio: int):
        """(hashes, starts, stops) of the last makeindex of the species."""
        nc = [d // grid_ratio for d in self.n]
        H = (nc[0] + 2) * (nc[1] + 2) * (nc[2] + 2)
        n = int(self.cfg.species[species].nvalid)
        hashes, starts, stops = np.empty(n, np.int64), np.empty(H, np.int64), np.empty(H, np.int64)
        p = lambda a: a.ctypes.data_as(C.POINTER(C.c_int64))  # noqa: E731
        self._check(self.lib.lcs_particles_cellindex(self.handle, species, p(hashes), p(starts), p(stops)))
        return hashes, starts, stops

    def particles_stat(self, species: int, tau_eta: float, grid_ratio: int = 4, bin_size: int = 16,
                       search_cell_size: int = 2, contact_tolerance: float = 0.01, min_radius: float = 1.25e-4,
                       max_wavenumber: int = 128, nsamples: int = 64) -> dict:
        """`Particles.stat` (src/particles/stat.jl:113-151); reorders the species
        by cell (makeindex!).  Defaults: the reference's cfgs/N1024-1.lcs-yaml."""
        pc = _abi.ParticleStatConfig(grid_ratio=grid_ratio, bin_size=bin_size, search_cell_size=search_cell_size,
                                     max_wavenumber=max_wavenumber, nsamples=nsamples,
                                     contact_tolerance=contact_tolerance, min_radius=min_radius)
        out = _abi.ParticleStats()
        self._check(self.lib.lcs_particles_stat(self.handle, species, C.byref(pc), float(tau_eta), C.byref(out)))
        return out.as_dict()

    def particles_density(self, species: int, grid_ratio: int) -> np.ndarray:
        """`Particles.density` (src/particles/stat.jl:176-215), in the new device order."""
        out = np.empty(int(self.cfg.species[species].nvalid))
        self._check(self.lib.lcs_particles_density(self.handle, species, grid_ratio, _dptr(out)))
        return out

    def flow_divergence(self):
        """(RMS, max |div|) of the current velocity over the interior cells."""
        r, m = C.c_double(), C.c_double()
        self._check(self.lib.lcs_flow_divergence(self.handle, C.byref(r), C.byref(m)))
        return r.value, m.value

    def flow_stat(self) -> dict:
        """`Flows.stat` (src/flows/stat.jl:66-153) computed on the device."""
        st = _abi.FlowStat()
        self._check(self.lib.lcs_flow_stat(self.handle, C.byref(st)))
        return st.as_dict()

    def step_timed(self, nsteps: int, logs: bool = True):
        """`step`, returning (logs, device milliseconds of the nsteps)."""
        arr = (_abi.Log * max(1, nsteps))() if logs else None
        ms = C.c_double()
        self._check(self.lib.lcs_step_timed(self.handle, nsteps, arr if logs else None, C.byref(ms)))
        return ([arr[q].as_dict() for q in range(nsteps)] if logs else None), ms.value

    def transfer_stats(self):
        """(host->device bytes, device->host bytes) copied by this handle so far."""
        a, b = C.c_int64(), C.c_int64()
        self._check(self.lib.lcs_transfer_stats(self.handle, C.byref(a), C.byref(b)))
        return a.value, b.value

    # -- stage functions ----------------------------------------------------
    def synchalo(self, fields, r: int, full: bool = True):
        """`Topologies.synchalo!` single process (lib/topologies/src/halo.jl:138-159)."""
        mask = 0
        for f in fields:
            mask |= 1 << f
        self._check(self.lib.lcs_synchalo(self.handle, mask, r, int(full)))

    def rhs(self, stage: int):
        """`Flows.rhs!` (src/flows/rhs.jl:20-42)."""
        self._check(self.lib.lcs_flow_rhs(self.handle, stage))

    def update(self, stage: int, dtrk: float):
        """`Flows.update!` (src/flows/update.jl:23-54)."""
        self._check(self.lib.lcs_flow_update(self.handle, stage, dtrk))

    def rhs_update(self, stage: int, dtrk: float):
        self._check(self.lib.lcs_flow_rhs_update(self.handle, stage, dtrk))

    def couple(self, stage: int, dtrk: float) -> dict:
        """`Flows.couple!(::HSMAC)` (src/flows/couples/hsmac.jl:52-75)."""
        log = _abi.CoupleLog()
        self._check(self.lib.lcs_flow_couple(self.handle, stage, dtrk, C.byref(log)))
        return {"itr": log.itr, "sweeps": log.sweeps, "div": log.div}

    def forcing(self, dtrk: float) -> dict:
        """`Flows.forcing!` (src/flows/forcings)."""
        p = C.c_double()
        e = C.c_double()
        self._check(self.lib.lcs_flow_forcing(self.handle, dtrk, C.byref(p), C.byref(e)))
        return {"p": p.value, "e10": e.value}

    def flow_timestep(self) -> float:
        """`Flows.timestep` (src/flows/timestep.jl:18-65)."""
        dt = C.c_double()
        self._check(self.lib.lcs_flow_timestep(self.handle, C.byref(dt)))
        return dt.value

    def particles_timestep(self) -> float:
        """`Particles.timestep` (src/particles/timestep.jl:6-25)."""
        dt = C.c_double()
        self._check(self.lib.lcs_particles_timestep(self.handle, C.byref(dt)))
        return dt.value

    def particles_boundary(self, species: int, stage: int):
        self._check(self.lib.lcs_particles_boundary(self.handle, species, stage))

    def particles_motion(self, species: int, stage: int):
        self._check(self.lib.lcs_particles_motion(self.handle, species, stage))

    def particles_update(self, species: int, stage: int, dtrk: float):
        self._check(self.lib.lcs_particles_update(self.handle, species, stage, dtrk))

    def init_particle_velocity(self, species: int):
        self._check(self.lib.lcs_init_particle_velocity(self.handle, species))

    # -- profiling ------------------------------------------------------------
    def profile(self, on: bool = True):
        self._check(self.lib.lcs_profile_enable(self.handle, int(on)))

    def profile_reset(self):
        self._check(self.lib.lcs_profile_reset(self.handle))

    def profile_totals(self) -> dict:
        """{kernel label: (total ms, launches)} since the last reset."""
        n = C.c_int32()
        self._check(self.lib.lcs_profile_count(self.handle, C.byref(n)))
        out = {}
        buf = C.create_string_buffer(128)
        for i in range(n.value):
            ms = C.c_double()
            cnt = C.c_int64()
            self._check(self.lib.lcs_profile_entry(self.handle, i, buf, 128, C.byref(ms), C.byref(cnt)))
            out[buf.value.decode()] = (ms.value, cnt.value)
        return out

    def launch_count(self) -> int:
        n = C.c_int64()
        self._check(self.lib.lcs_launch_count(self.handle, C.byref(n)))
        return n.value

    def synchronize(self):
        self._check(self.lib.lcs_synchronize(self.handle))


def footprint(cfg: _abi.Config) -> int:
    """Device bytes a handle of this config holds (serving admission)."""
    lib = _abi.load_library()
    b = C.c_int64()
    rc = lib.lcs_footprint(C.byref(cfg), C.byref(b))
    if rc != 0:
        raise LCSError(rc, lib.lcs_last_error(None).decode())
    return b.value
