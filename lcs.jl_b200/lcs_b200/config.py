"""`.lcs-yaml` configuration -> the C ABI's ``lcs_config``.

The YAML schema is the reference's (kind-tagged ``{"kind": ..., "params":
...}`` objects, lib/polyserde/src/PolySerde.jl:35-80; field names of
src/config.jl, src/flows/config.jl, src/particles/config.jl).  The backend kind
``b200`` is new; its optional params are ``precision`` ("fp64" or
"fp32-mixed"), ``device``, ``graphs`` and ``particle_sort`` (sort the particles
by cell every that many steps: lcs_set_particle_sort with the first species'
cell grid_ratio; 0 or absent: off).

New init kinds (no reference counterpart, generated on the host):
  flow.init "spectral"      params {seed, urms, kpeak}
  particles.init.velocity "interp"  (fluid velocity at the particle)
  particles.init.position "random"  params {seed} (optional seed)
"""

from __future__ import annotations

import copy
import math
from dataclasses import dataclass, field

from . import _abi

COLORINGS = {
    "no": _abi.COLORING_NO,
    "red-black": _abi.COLORING_RED_BLACK,
    "red-black-fast": _abi.COLORING_RED_BLACK_FAST,
    "red-black-block": _abi.COLORING_RED_BLACK_BLOCK,
}
FORCINGS = {"no": _abi.FORCING_NO, "linear-power": _abi.FORCING_LINEAR_POWER, "rc-energy": _abi.FORCING_RC_ENERGY}
DRAGS = {"linear": _abi.DRAG_LINEAR, "nonlinear": _abi.DRAG_NONLINEAR}
MODES = {"flow": _abi.MODE_FLOW, "flow-particle": _abi.MODE_FLOW_PARTICLE}
PRECISIONS = {"fp64": _abi.PRECISION_FP64, "fp32-mixed": _abi.PRECISION_FP32_MIXED}


def _kind(x, default=None):
    if x is None:
        return default, {}
    if isinstance(x, str):
        return x, {}
    return x.get("kind", default), (x.get("params") or {})


@dataclass
class SpeciesInit:
    """Host-side particle init of one species (src/particles/init.jl)."""

    nvalid: int
    diam: float                     # non-dimensional diameter diam_m / L0 (particles/config.jl:233)
    position: str = "random"
    position_seed: int = 0
    velocity: str = "rest"          # "rest" | "interp" | "restart"
    id_kind: str = "generate"       # "generate" | "restart"
    size: str = "const"             # "const" | "restart"
    restart_file: str = ""          # ParticleRestart(file, iprofile) of any "restart" kind
    restart_profile: int = 0
    # Cell, RDF and Spectrum of the species' statistics (particles/config.jl:51-108)
    grid_ratio: int = 4
    rdf: dict = field(default_factory=lambda: {"contact_tolerance": 0.01, "bin_size": 16, "min_radius": 1.0e-3,
                                               "search_cell_size": 1})
    spectrum: dict = field(default_factory=lambda: {"max_wavenumber": 128, "nsamples": 64})


@dataclass
class RunConfig:
    """What `LCS.simulate` needs beyond the C struct."""

    abi: _abi.Config
    flow_init: str
    flow_init_params: dict
    species: list = field(default_factory=list)
    last_step: int = 0
    interval_stat: int = 1
    particle_sort: int = 0          # backend param: lcs_set_particle_sort interval (0: off)
    interval_restart: int = 0       # 0: no restart files
    num_restart_files: int = 1
    outdir: str = "output"
    raw: dict = field(default_factory=dict)

    @property
    def dims(self):
        return tuple(int(d) for d in self.abi.dims)


def from_dict(d: dict) -> RunConfig:
    """Deserialize a reference config dict (LCSIO.readconfig output)."""
    d = copy.deepcopy(d)
    c = _abi.Config()
    c.abi_version = _abi.ABI_VERSION
    mode, _ = _kind(d.get("mode"), "flow-particle")
    c.mode = MODES[mode]
    bkind, bparams = _kind(d.get("backend"), "b200")
    if bkind not in ("b200", "cuda", "cpu"):
        raise ValueError(f"unknown backend kind {bkind!r}")
    c.precision = PRECISIONS[bparams.get("precision", "fp64")]
    c.device = int(bparams.get("device", 0))
    c.use_graphs = int(bool(bparams.get("graphs", True)))
    grid = d["grid"]
    dims = list(grid["dims"])
    if len(dims) != 3:
        raise ValueError("grid.dims must have 3 entries")
    for a in range(3):
        c.dims[a] = int(dims[a])
    c.halo_size = int(grid.get("halo_size", 3))
    ts = d["timestep"]
    c.cfl = float(ts["cfl"])
    c.dtmax = float(ts["dtmax"])
    flow = d["flow"]
    fp = flow["params"]
    c.U0, c.L0, c.NU = float(fp["U0_m_s"]), float(fp["L0_m"]), float(fp["NU_m2_s"])
    ck, cp = _kind(flow["couple"], "hsmac")
    if ck != "hsmac":
        raise ValueError(f"unsupported couple kind {ck!r} (the reference implements only hsmac)")
    c.time_blocking = int(bool(cp["time_blocking"]))
    c.overlap = int(bool(cp["overlap"]))
    colk, colp = _kind(cp["coloring"], "red-black-fast")
    c.coloring = COLORINGS[colk]
    c.coloring_block = int(colp.get("size", 0))
    c.omega = float(cp["omega"])
    c.epsp = float(cp["epsp"])
    c.itrmin = int(cp["itrmin"])
    c.itrmax = int(cp["itrmax"])
    fk, fpp = _kind(flow.get("forcing"), "no")
    c.forcing = FORCINGS[fk]
    if fk == "linear-power":
        c.power = float(fpp["power"])
    elif fk == "rc-energy":
        c.energy = float(fpp["energy"])
        c.kmin, c.kmax, c.coarse_size = int(fpp["kmin"]), int(fpp["kmax"]), int(fpp["coarse_size"])
    ik, ip = _kind(flow.get("init"), "spectral")
    species = []
    parts = d.get("particles") or []
    if c.mode == _abi.MODE_FLOW_PARTICLE:
        if len(parts) > _abi.MAX_SPECIES:
            raise ValueError(f"at most {_abi.MAX_SPECIES} particle species")
        c.n_species = len(parts)
        for s, pc in enumerate(parts):
            pop = pc["population"]
            nvalid = int(pop["valid"])
            c.species[s].nvalid = nvalid
            pp = pc["params"]
            c.species[s].gravity = float(pp["gravity"])
            c.species[s].density_ratio = float(pp["density_ratio"])
            dk, _ = _kind(pc.get("drag"), "linear")
            c.species[s].drag = DRAGS[dk]
            init = pc.get("init") or {}
            sk, sp = _kind(init.get("size"), "const")
            if sk not in ("const", "restart"):
                raise ValueError(f"unsupported particle size init {sk!r}")
            diam = float(sp["diam_m"]) / c.L0 if sk == "const" else 0.0
            pk, pp2 = _kind(init.get("position"), "random")
            vk, vp = _kind(init.get("velocity"), "rest")
            idk, idp = _kind(init.get("id"), "generate")
            si = SpeciesInit(nvalid=nvalid, diam=diam, position=pk, position_seed=int(pp2.get("seed", 1000 + s)),
                             velocity=vk, id_kind=idk, size=sk)
            for k, prm in ((pk, pp2), (vk, vp), (idk, idp), (sk, sp)):  # ParticleRestart (particles/config.jl:150-153)
                if k == "restart":
                    si.restart_file = str(prm["file"])
                    si.restart_profile = int(prm.get("iprofile", s + 1))
            si.grid_ratio = int((pc.get("cell") or {}).get("grid_ratio", si.grid_ratio))
            st = pc.get("stat") or {}
            si.rdf.update(st.get("rdf") or {})
            si.spectrum.update(st.get("spectrum") or {})
            species.append(si)
    sim = d.get("simulate") or {}
    return RunConfig(abi=c, flow_init=ik, flow_init_params=ip, species=species,
                     last_step=int(sim.get("last_step", 0)), interval_stat=int(sim.get("interval_stat", 1)),
                     interval_restart=int(sim.get("interval_restart", 0)),
                     num_restart_files=int(sim.get("num_restart_files", 1)), outdir=str(d.get("outdir", "output")),
                     particle_sort=int(bparams.get("particle_sort", 0) or 0), raw=d)


def readconfig(path: str) -> RunConfig:
    """`LCSIO.readconfig` (src/LCSIO/config.jl:6-31) for a `.lcs-yaml` file."""
    import yaml

    with open(path) as f:
        return from_dict(yaml.safe_load(f))


def taup(density_ratio: float, Re: float, diam: float) -> float:
    """`Particles.taup` (src/particles/config.jl:41)."""
    return 1.0 / 18.0 * density_ratio * Re * (diam * diam)


def diam_for_taup(tp: float, density_ratio: float, Re: float) -> float:
    """Non-dimensional diameter giving a Stokes time tp."""
    return math.sqrt(18.0 * tp / (density_ratio * Re))


def workload(n: int, nu: float, forcing: dict, taups: list, counts: list, *, epsp_rms: float = 1e-8,
             seed: int = 0, precision: str = "fp64", itrmax: int = 300, steps: int = 100,
             density_ratio: float = 843.0) -> dict:
    """A reference-format config dict for a synthetic turbulence workload.

    L = 2pi, U0 = L0 = 1 (Re = 1/nu); spectral init E(k) ~ k^4 exp(-2(k/4)^2)
    with u_rms = 1; HSMAC red-black-fast with time blocking and overlap (the
    production settings of cfgs/*.lcs-yaml), omega 1.7, itrmin 6, and epsp =
    epsp_rms * dxmin so the exit test reads RMS(div) < epsp_rms; linear (Stokes)
    drag, g = 0, particle velocity = interpolated fluid velocity.
    """
    Re = 1.0 / nu
    dx = 2.0 * math.pi / n
    parts = []
    for s, (tp, cnt) in enumerate(zip(taups, counts)):
        parts.append({
            "population": {"valid": int(cnt), "invalid_ratio": 0.0, "exchange_ratio": 0.0},
            "params": {"gravity": 0.0, "density_ratio": density_ratio},
            "cell": {"grid_ratio": 4},
            "drag": {"kind": "linear"},
            "init": {
                "id": {"kind": "generate"},
                "position": {"kind": "random", "params": {"seed": seed * 1000 + 17 + s}},
                "velocity": {"kind": "interp"},
                "size": {"kind": "const", "params": {"diam_m": diam_for_taup(tp, density_ratio, Re)}},
            },
        })
    return {
        "outdir": "output",
        "mode": {"kind": "flow-particle" if parts else "flow"},
        "backend": {"kind": "b200", "params": {"precision": precision}},
        "topo": {"proc_dims": [0, 0, 0], "reorder": False},
        "grid": {"dims": [n, n, n], "halo_size": 3},
        "timestep": {"cfl": 0.3, "dtmax": 0.01},
        "simulate": {"last_step": steps, "interval_stat": steps, "interval_restart": 10**9, "interval_gc": 1000,
                     "num_restart_files": 1},
        "flow": {
            "params": {"U0_m_s": 1.0, "L0_m": 1.0, "NU_m2_s": nu},
            "init": {"kind": "spectral", "params": {"seed": seed, "urms": 1.0, "kpeak": 4.0}},
            "couple": {"kind": "hsmac", "params": {
                "time_blocking": True, "overlap": True, "coloring": {"kind": "red-black-fast"},
                "omega": 1.7, "epsp": epsp_rms * dx, "itrmin": 6, "itrmax": itrmax}},
            "forcing": forcing,
            "stat": {"integral_length": False},
        },
        "particles": parts,
    }
