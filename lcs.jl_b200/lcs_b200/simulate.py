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
    from . import restart

    eng = engine_cls(rc.abi)
    n = rc.dims[0]
    if rc.flow_init in ("restart", "upsample"):  # LCS.Restart / Upsample (flows/inits/init.jl:16-24)
        f = str(rc.flow_init_params["file"])
        if rc.flow_init == "restart":
            U, V, W, P = (restart.dataset(eng.lib, f, "flow/" + c) for c in "UVWP")
            eng.upload_flow(U, V, W, P)
        else:
            restart.load_coarse(eng, f)
    elif rc.flow_init == "spectral":
        p = rc.flow_init_params
        U, V, W, P = inits.spectral_flow(n, seed=int(p.get("seed", 0)), urms=float(p.get("urms", 1.0)),
                                         kpeak=float(p.get("kpeak", 4.0)))
    elif rc.flow_init == "ideal-flow":
        U, V, W, P = inits.ideal_flow(n)
    else:
        raise ValueError(f"flow init {rc.flow_init!r} is not available on the B200 backend "
                         "(random-flow needs Julia's Xoshiro stream)")
    if rc.flow_init in ("spectral", "ideal-flow"):
        eng.upload_flow(U, V, W, P)
    offset = 0
    for s, si in enumerate(rc.species):
        # ParticleRestart (particles/config.jl:150-217): particles/<iprofile>/... of a restart file
        def from_file(name, si=si):
            a = restart.dataset(eng.lib, si.restart_file, f"particles/{si.restart_profile}/{name}")
            if a.size != si.nvalid:
                raise ValueError(f"{si.restart_file}: particles/{si.restart_profile}/{name} holds {a.size} "
                                 f"particles, the species {si.nvalid}")
            return a.reshape(-1)
        if si.position == "restart":
            x, y, z = from_file("x"), from_file("y"), from_file("z")
        elif si.position == "random":
            x, y, z = inits.random_positions(si.nvalid, si.position_seed)
        else:
            raise ValueError(f"particle position init {si.position!r} is not available")
        zeros = np.zeros(si.nvalid)
        u, v, w = (from_file(c) for c in "uvw") if si.velocity == "restart" else (zeros, zeros, zeros)
        diam = from_file("diam") if si.size == "restart" else np.full(si.nvalid, si.diam)
        ids = from_file("id") if si.id_kind == "restart" else inits.generate_ids(si.nvalid, offset)
        offset += si.nvalid
        eng.upload_particles(s, diam, x, y, z, u, v, w, ids=ids)
        if si.velocity == "interp":
            eng.init_particle_velocity(s)
        elif si.velocity not in ("rest", "restart"):
            raise ValueError(f"particle velocity init {si.velocity!r} is not available")
    if rc.particle_sort > 0 and rc.species:
        eng.set_particle_sort(rc.particle_sort, rc.species[0].grid_ratio)
    return eng


def latest_restart(outdir: str):
    """LCSIO.find_latest_restart_file (LCSIO/config.jl:105-120): the
    restart.h5.<step> of the largest step, and that step; (None, 0) if none."""
    import os
    import re

    best, step = None, -1
    if os.path.isdir(outdir):
        for f in os.listdir(outdir):
            m = re.fullmatch(r"restart\.h5\.(\d+)", f)
            if m and int(m.group(1)) > step:
                best, step = os.path.join(outdir, f), int(m.group(1))
    return best, max(step, 0)


def patch_resume(rc: RunConfig, file: str) -> RunConfig:
    """LCSIO.patch_resume (LCSIO/config.jl:80-101): every init reads the restart file."""
    import copy

    rc = copy.copy(rc)
    rc.flow_init, rc.flow_init_params = "restart", {"file": file}
    rc.species = [copy.copy(si) for si in rc.species]
    for s, si in enumerate(rc.species):
        si.position = si.velocity = si.id_kind = si.size = "restart"
        si.restart_file, si.restart_profile = file, s + 1
    return rc


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
             outdir: str | None = None, resume: bool | None = None):
    """Run the configured simulation; returns (engine, logs).

    With save=True, as `LCS.simulate` does through LCSIO: every interval_stat
    steps the statistics go into `<outdir>/stat.h5` (one group per step), and
    every interval_restart steps the state into `<outdir>/restart.h5.<step>`,
    keeping the last num_restart_files of them (LCSIO.cleanrestart).

    resume (default with save=True: the LCS_RESUME environment variable, as
    LCSIO.init reads it; otherwise False): continue from the latest
    restart.h5.<step> in outdir, with t from stat.h5
    (LCSIO.load_resume_state!).  Without `steps`, the run takes the
    reference's last_step - step + 1 steps (its loop over state.step:last_step),
    ending at step last_step + 1."""
    import os

    from . import restart

    rc = config if isinstance(config, RunConfig) else (readconfig(config) if isinstance(config, str) else from_dict(config))
    out = outdir or rc.outdir
    if resume is None:  # the environment decides only for runs that write their outputs
        resume = save and os.environ.get("LCS_RESUME", "0").lower() in ("1", "true", "yes")
    start = 0
    if resume:
        file, start = latest_restart(out)
        if file is None:
            raise ValueError(f"no restart files to resume from in {out}")
        rc = patch_resume(rc, file)
    eng = init_engine(rc, engine_cls)
    if resume:
        t, _ = restart.load_state(eng.lib, os.path.join(out, "stat.h5"), start)
        eng.set_state(start, t)
    # the reference loops `for _ in state.step:last_step` (src/simulate.jl:54):
    # last_step - step + 1 steps, so a fresh run ends at step last_step + 1
    last = (rc.last_step - start + 1) if steps is None else steps
    istat = max(1, rc.interval_stat)
    irest = rc.interval_restart if save else 0
    if save:
        os.makedirs(out, exist_ok=True)
    logs = []
    done = 0
    while done < last:
        # up to the next statistics (or restart) step, device-resident in between
        at = start + done
        chunk = min(istat - at % istat, last - done)
        if irest > 0:
            chunk = min(chunk, irest - at % irest)
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


def main(argv=None, engine_cls=Engine):
    """`julia simulate.jl cfg.lcs-yaml` equivalent: python -m lcs_b200 cfg.lcs-yaml [steps].

    As LCSIO.init does (LCSIO/config.jl:30-76): a fresh run needs a new output
    directory and saves the config there as config.lcs-yaml; an existing one
    is resumed only with LCS_RESUME=1, and only if it holds restart files and
    that config.  Statistics and restart files are written at their intervals."""
    import os

    import yaml

    argv = sys.argv[1:] if argv is None else argv
    if not argv:
        print("usage: python -m lcs_b200 <config.lcs-yaml> [steps]", file=sys.stderr)
        return 2
    steps = int(argv[1]) if len(argv) > 1 else None
    rc = readconfig(argv[0])
    out = rc.outdir
    resume = os.environ.get("LCS_RESUME", "0").lower() in ("1", "true", "yes")
    if os.path.isdir(out):
        if not resume:
            raise ValueError(f"output directory {out} already exists, set LCS_RESUME=1 to resume")
        if latest_restart(out)[0] is None or not os.path.isfile(os.path.join(out, "config.lcs-yaml")):
            raise ValueError(f"output directory {out} exists but is not resumable, "
                             "missing restart files or config.lcs-yaml")
    else:
        resume = False
        os.makedirs(out)
        with open(os.path.join(out, "config.lcs-yaml"), "w") as f:
            yaml.safe_dump(rc.raw, f, sort_keys=False)
    eng, _ = simulate(rc, steps=steps, engine_cls=engine_cls, save=True, outdir=out, resume=resume)
    eng.close()
    return 0


__all__ = ["simulate", "init_engine", "main", "_abi"]
