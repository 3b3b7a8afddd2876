"""CUDA library against the oracle on the two plain-FP64 workloads at full size.

- lp128: 128^3, nu 0.01, linear-power P = 0.5, 65,536 Stokes particles
  (tau_p 0.1), HSMAC red-black-fast with time blocking and overlap, itrmax 300,
  RMS(div) < 1e-8, 10 steps.
- rc256: 256^3, nu 0.005, rc-energy with a 16-cell box filter (coarse 16^3),
  2^20 particles in 2 species (tau_p 0.05, 0.5), 10 steps.

Both start from the same seeded host inputs.  After 10 steps (the stage order
of src/evolve.jl:63-146) the velocity and pressure fields must agree to
relative L2 <= 1e-10, the HSMAC sweep count of every couple must be equal, and
the particles must agree to relative L2 <= 1e-10.  Particle cell and index
assignment is integer work and must be bit-exact given identical positions:
the oracle's final state is loaded into both libraries and the interpolation
mapping (src/particles/interp.jl:92-126, through motion! with linear drag)
and the cell hashes, starts and stops of makeindex!
(src/particles/makeindex.jl:29-67) are compared with `==`.
"""

import numpy as np
import pytest

from helpers import rel_l2
from lcs_b200 import Engine
from lcs_b200 import _abi as F
from lcs_b200 import workloads as wl
from oracle_engine import OracleEngine

pytestmark = pytest.mark.gpu

STEPS = 10


def run_both(name):
    rc, w = wl.make_run_config(name)
    flow, parts = wl.host_inputs(rc)
    out = {}
    for cls, graphs in ((Engine, 1), (OracleEngine, 0)):
        rc.abi.use_graphs = graphs
        e = cls(rc.abi)
        wl.load_engine(e, rc, flow, parts)
        if graphs:
            logs = e.step(STEPS)  # the device-resident step graphs of the product path
        else:
            logs = []
            for _ in range(STEPS):
                dt = e.timestep()
                logs.append(e.evolve(dt))
        out[cls] = (e, logs)
    return rc, out[Engine], out[OracleEngine]


def check_steps(rc, gpu, orc):
    (g, lg), (o, lo) = gpu, orc
    assert len(lg) == len(lo) == STEPS
    for a, b in zip(lg, lo):
        for c in ("couple1", "couple2"):
            assert a[c]["itr"] == b[c]["itr"], (c, a[c], b[c])
            assert abs(a[c]["div"] - b[c]["div"]) <= 1e-9 * b[c]["div"]
        assert abs(a["dt"] - b["dt"]) <= 1e-12 * b["dt"]
        assert abs(a["forcing"]["p"] - b["forcing"]["p"]) <= 1e-9 * abs(b["forcing"]["p"])
    fg, fo = g.download_flow(), o.download_flow()
    for name, a, b in zip("UVWP", fg, fo):
        assert rel_l2(a, b) <= 1e-10, (name, rel_l2(a, b))
    parts_o = []
    for s in range(len(rc.species)):
        pg, po = g.download_particles(s), o.download_particles(s)
        assert np.array_equal(pg["ids"], po["ids"])
        for k in ("x", "y", "z", "u", "v", "w"):
            assert rel_l2(pg[k], po[k]) <= 1e-10, (s, k, rel_l2(pg[k], po[k]))
        parts_o.append(po)
    assert g.get_state()[0] == o.get_state()[0] == STEPS
    return fo, parts_o


def check_assignment(rc, g, o, fo, parts_o):
    """Identical positions and fields in both libraries: the interpolation of
    motion! and the cell index are bit-exact."""
    for e in (g, o):
        e.upload_flow(*fo)
        # motion! reads the halo that evolve!'s FullHalo synchalo! fills first (src/evolve.jl:74-81)
        e.synchalo([F.FIELD_U, F.FIELD_V, F.FIELD_W], 3, True)
        for s, po in enumerate(parts_o):
            e.upload_particles(s, po["diam"], po["x"], po["y"], po["z"], po["u"], po["v"], po["w"], ids=po["ids"])
    for s in range(len(parts_o)):
        g.particles_motion(s, 1)
        o.particles_motion(s, 1)
        for p in (F.PROP_DUDT, F.PROP_DVDT, F.PROP_DWDT):
            assert np.array_equal(g.prop_get(s, p), o.prop_get(s, p)), (s, F.PROP_NAMES[p])
        ratio = rc.species[s].grid_ratio
        g.particles_makeindex(s, 1, ratio)
        o.particles_makeindex(s, 1, ratio)
        for name, a, b in zip(("hashes", "starts", "stops"), g.particles_cellindex(s, ratio),
                              o.particles_cellindex(s, ratio)):
            assert np.array_equal(a, b), (s, name)
        # the stable sort leaves both libraries with the same particle order
        assert np.array_equal(g.download_particles(s)["ids"], o.download_particles(s)["ids"])


@pytest.mark.parametrize("name", ["lp128", "rc256"])
def test_workload_ten_steps(name):
    rc, gpu, orc = run_both(name)
    try:
        fo, parts_o = check_steps(rc, gpu, orc)
        check_assignment(rc, gpu[0], orc[0], fo, parts_o)
    finally:
        gpu[0].close()
        orc[0].close()
