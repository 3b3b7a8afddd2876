"""`LCS.simulate(config)` on the B200 backend (src/simulate.jl:13-90).

Setup (buffers, state, init) happens on the host; every step then calls the
two per-step entry points `timestep!` and `evolve!`, which run entirely on the
GPU.  Between statistics intervals the steps are issued as device-resident
CUDA graphs (`lcs_step`), so the host does not touch the GPU per step.
"""

from __future__ import annotations

import sys

import numpy as np

from . import _abi, inits
from .config import RunConfig, from_dict, readconfig
from .engine import Engine


def init_engine(rc: RunConfig, engine_cls=Engine) -> Engine:
    """`LCS.Buffer` + `LCS.State` + `LCS.init!` (src/init.jl:6-26)."""
    eng = engine_cls(rc.abi)
    n = rc.dims[0]
    if rc.flow_init == "spectral":
        p = rc.flow_init_params
        U, V, W, P = inits.spectral_flow(n, seed=int(p.get("seed", 0)), urms=float(p.get("urms", 1.0)),
                                         kpeak=float(p.get("kpeak", 4.0)))
    elif rc.flow_init == "ideal-flow":
        U, V, W, P = inits.ideal_flow(n)
    else:
        raise ValueError(f"flow init {rc.flow_init!r} is not available on the B200 backend "
                         "(random-flow needs Julia's Xoshiro stream; restart/upsample need HDF5)")
    eng.upload_flow(U, V, W, P)
    offset = 0
    for s, si in enumerate(rc.species):
        if si.position != "random":
            raise ValueError(f"particle position init {si.position!r} is not available")
        x, y, z = inits.random_positions(si.nvalid, si.position_seed)
        zeros = np.zeros(si.nvalid)
        diam = np.full(si.nvalid, si.diam)
        ids = inits.generate_ids(si.nvalid, offset)
        offset += si.nvalid
        eng.upload_particles(s, diam, x, y, z, zeros, zeros, zeros, ids=ids)
        if si.velocity == "interp":
            eng.init_particle_velocity(s)
        elif si.velocity != "rest":
            raise ValueError(f"particle velocity init {si.velocity!r} is not available")
    return eng


def printstate(step: int, t: float, dt: float, log: dict, out=None):
    """`LCS.printstate` + `printlog` (src/stat.jl:48-85), one line per step
    (to `out`, by default the current sys.stdout)."""
    c1, c2 = log["couple1"], log["couple2"]
    (out or sys.stdout).write(f"step={step} t={t:.6e} dt={dt:.6e} couple1=(itr={c1['itr']}, div={c1['div']:.3e}) "
                              f"couple2=(itr={c2['itr']}, div={c2['div']:.3e}) p={log['forcing']['p']:.6e}\n")


def save_stat(eng, rc: RunConfig, log: dict, path: str):
    """`LCS.stat` + `LCSIO.savestat` (src/simulate.jl:62-66): Flows.stat and
    Particles.stat of every species on the device, written as the step's entry
    of the stat file (the species are reordered by cell, as in the reference)."""
    import ctypes as C

    from . import restart

    fs = eng.flow_stat()
    pstats = []
    for s, si in enumerate(rc.species):
        pc = _abi.ParticleStatConfig(grid_ratio=si.grid_ratio, bin_size=int(si.rdf["bin_size"]),
                                     search_cell_size=int(si.rdf["search_cell_size"]),
                                     max_wavenumber=int(si.spectrum["max_wavenumber"]),
                                     nsamples=int(si.spectrum["nsamples"]),
                                     contact_tolerance=float(si.rdf["contact_tolerance"]),
                                     min_radius=float(si.rdf["min_radius"]))
        ps = _abi.ParticleStats()
        eng._check(eng.lib.lcs_particles_stat(eng.handle, s, C.byref(pc), float(fs["tau_eta"]), C.byref(ps)))
        pstats.append(ps)
    lg = _abi.Log()
    for k in ("couple1", "couple2"):
        getattr(lg, k).itr, getattr(lg, k).sweeps, getattr(lg, k).div = (log[k]["itr"], log[k]["sweeps"],
                                                                          log[k]["div"])
    lg.forcing_p, lg.forcing_e10 = log["forcing"]["p"], log["forcing"]["e10"]
    lg.dt, lg.t, lg.step = log["dt"], log["t"], log["step"]
    restart.save_stat(eng.lib, path, int(log["step"]), float(log["t"]), float(log["dt"]), flow=fs,
                      nvalid=[si.nvalid for si in rc.species] or None, particles=pstats or None, log=lg)


def simulate(config, *, steps: int | None = None, quiet: bool = False, engine_cls=Engine, save: bool = False,
             outdir: str | None = None):
    """Run the configured simulation; returns (engine, logs).

    With save=True, as `LCS.simulate` does through LCSIO: every interval_stat
    steps the statistics go into `<outdir>/stat.h5` (one group per step), and
    every interval_restart steps the state into `<outdir>/restart.h5.<step>`,
    keeping the last num_restart_files of them (LCSIO.cleanrestart)."""
    import os

    from . import restart

    rc = config if isinstance(config, RunConfig) else (readconfig(config) if isinstance(config, str) else from_dict(config))
    eng = init_engine(rc, engine_cls)
    last = rc.last_step if steps is None else steps
    istat = max(1, rc.interval_stat)
    irest = rc.interval_restart if save else 0
    out = outdir or rc.outdir
    if save:
        os.makedirs(out, exist_ok=True)
    logs = []
    done = 0
    while done < last:
        # up to the next statistics (or restart) step, device-resident in between
        chunk = min(istat - done % istat, last - done)
        if irest > 0:
            chunk = min(chunk, irest - done % irest)
        for lg in eng.step(chunk):
            logs.append(lg)
            if not quiet:
                printstate(lg["step"], lg["t"], lg["dt"], lg)
        done += chunk
        step = int(logs[-1]["step"])
        if save and step % istat == 0:
            save_stat(eng, rc, logs[-1], os.path.join(out, "stat.h5"))
        if irest > 0 and step % irest == 0:
            restart.save(eng, os.path.join(out, f"restart.h5.{step}"))
            old = os.path.join(out, f"restart.h5.{step - irest * rc.num_restart_files}")
            if os.path.isfile(old):
                os.remove(old)
    return eng, logs


def main(argv=None):
    """`julia simulate.jl cfg.lcs-yaml` equivalent: python -m lcs_b200 cfg.lcs-yaml"""
    argv = sys.argv[1:] if argv is None else argv
    if not argv:
        print("usage: python -m lcs_b200 <config.lcs-yaml> [steps]", file=sys.stderr)
        return 2
    steps = int(argv[1]) if len(argv) > 1 else None
    simulate(argv[0], steps=steps)
    return 0


__all__ = ["simulate", "init_engine", "main", "_abi"]
