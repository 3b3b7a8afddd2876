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


def simulate(config, *, steps: int | None = None, quiet: bool = False, engine_cls=Engine):
    """Run the configured simulation; returns (engine, logs)."""
    rc = config if isinstance(config, RunConfig) else (readconfig(config) if isinstance(config, str) else from_dict(config))
    eng = init_engine(rc, engine_cls)
    last = rc.last_step if steps is None else steps
    interval = max(1, rc.interval_stat)
    logs = []
    done = 0
    while done < last:
        chunk = min(interval, last - done)
        for lg in eng.step(chunk):
            logs.append(lg)
            if not quiet:
                printstate(lg["step"], lg["t"], lg["dt"], lg)
        done += chunk
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
