"""The synthetic turbulence workloads the backend is measured and checked on.

Each is a reference-format config (`config.workload`) plus its seeded host
inputs: the solenoidal spectral velocity field E(k) ~ k^4 exp(-2(k/4)^2) with
u_rms = 1, uniform random particle positions, and particle velocity equal to
the interpolated fluid velocity.  The reference has no such inits (its
random-flow uses Julia's Xoshiro stream); they are generated here once and
fed identically to the CUDA library and to the oracle.
"""

from __future__ import annotations

import numpy as np

from . import config as lcfg
from . import inits

LINEAR_POWER = {"kind": "linear-power", "params": {"power": 0.5}}
# rc-energy with a 16-cell box filter at 256^3 (coarse 16^3); kmin, kmax and the
# energy come from the reference's cfgs/N256.lcs-yaml
RC_ENERGY_16 = {"kind": "rc-energy", "params": {"kmin": 1, "kmax": 2, "energy": 0.649, "coarse_size": 16}}

WORKLOADS = {
    # plain FP64, 128^3, nu 0.01, linear-power P = 0.5, 65,536 particles tau_p = 0.1
    "lp128": dict(n=128, nu=0.01, forcing=LINEAR_POWER, taups=[0.1], counts=[65536], precision="fp64"),
    # plain FP64, 256^3, nu 0.005, rc-energy (16-cell filter), 2^20 particles in 2 species
    "rc256": dict(n=256, nu=0.005, forcing=RC_ENERGY_16, taups=[0.05, 0.5], counts=[2 ** 19, 2 ** 19],
                  precision="fp64"),
    # 512^3, nu 0.0025, linear-power P = 0.5, 2^24 particles in 3 species; run
    # in both precision forms (FP64 and FP32-mixed) from the same seed
    "lp512": dict(n=512, nu=0.0025, forcing=LINEAR_POWER, taups=[0.02, 0.2, 2.0],
                  counts=[2 ** 24 // 3, 2 ** 24 // 3, 2 ** 24 - 2 * (2 ** 24 // 3)], precision="fp64"),
}


def make_run_config(name, seed=0, precision=None, itrmax=300):
    """RunConfig and the workload's parameters."""
    w = WORKLOADS[name]
    d = lcfg.workload(w["n"], w["nu"], w["forcing"], w["taups"], w["counts"], seed=seed,
                      precision=precision or w["precision"], itrmax=itrmax)
    return lcfg.from_dict(d), w


def host_inputs(rc, pinned=False):
    """Seeded initial state on the host: ((U, V, W, P), [(diam, x, y, z) per
    species]), optionally in pinned (page-locked) memory."""
    n = rc.dims[0]
    p = rc.flow_init_params
    U, V, W, P = inits.spectral_flow(n, seed=int(p.get("seed", 0)), urms=float(p.get("urms", 1.0)),
                                     kpeak=float(p.get("kpeak", 4.0)))
    parts = []
    for si in rc.species:
        x, y, z = inits.random_positions(si.nvalid, si.position_seed)
        parts.append((np.full(si.nvalid, si.diam), x, y, z))
    if pinned:
        import torch

        def pin(a):
            t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
            t.numpy()[...] = a
            return t.numpy()

        U, V, W, P = (pin(a) for a in (U, V, W, P))
        parts = [tuple(pin(a) for a in sp) for sp in parts]
    return (U, V, W, P), parts


def load_engine(eng, rc, flow, parts):
    """Upload the state into a handle; particle velocity = interpolated fluid
    velocity where the species asks for it."""
    eng.upload_flow(*flow)
    for s, (d, x, y, z) in enumerate(parts):
        zero = np.zeros_like(x)
        eng.upload_particles(s, d, x, y, z, zero, zero, zero)
        if rc.species[s].velocity == "interp":
            eng.init_particle_velocity(s)
