"""CUDA library vs the CPU oracle on identical seeded inputs, stage by stage.

Element-wise stages compile without FMA contraction on both sides, so the
FP64 fields must agree bit for bit; quantities that pass through a mean
(forcing amplitudes, HSMAC residual) agree to 1e-12 relative, and after 10
full steps the fields agree to rel-L2 <= 1e-10, the plain method's parity bound.
"""

import math

import numpy as np
import pytest

from helpers import load_particles, load_random_flow, make_config, rel_l2
from lcs_b200 import Engine, _abi
from oracle_engine import OracleEngine

F = _abi
pytestmark = pytest.mark.gpu


def pair(cfg):
    return Engine(cfg), OracleEngine(cfg)


def same_fields(ea, eb, fields, haloed=False):
    for f in fields:
        a, b = ea.field_get(f, haloed=haloed), eb.field_get(f, haloed=haloed)
        assert np.array_equal(a, b), (F.FIELD_NAMES[f], np.abs(a - b).max())


@pytest.mark.parametrize("dims", [(16, 16, 16), (32, 32, 32), (18, 24, 20)])
@pytest.mark.parametrize("stage", [1, 2])
def test_rhs_bitwise(dims, stage):
    cfg = make_config(dims=dims, mode=F.MODE_FLOW, Re=7.0)
    g, o = pair(cfg)
    load_random_flow([g, o], seed=1, fields=(0, 1, 2, 3, 4, 5, 6))
    g.rhs(stage)
    o.rhs(stage)
    same_fields(g, o, (F.FIELD_DUDT, F.FIELD_DVDT, F.FIELD_DWDT))


@pytest.mark.parametrize("stage", [1, 2])
def test_update_and_fused_rhs_update_bitwise(stage):
    cfg = make_config(16, mode=F.MODE_FLOW, Re=3.0)
    g, o = pair(cfg)
    load_random_flow([g, o], seed=2, fields=(0, 1, 2, 3, 4, 5, 6))
    rng = np.random.default_rng(3)
    for f in (F.FIELD_DUDT, F.FIELD_DVDT, F.FIELD_DWDT):
        a = rng.random(g.interior_shape)
        g.field_set(f, a)
        o.field_set(f, a)
    g.update(stage, 0.01)
    o.update(stage, 0.01)
    same_fields(g, o, (0, 1, 2, 3, 4, 5))
    # fused: rhs! then update! in one pass equals the two reference kernels
    load_random_flow([g, o], seed=4, fields=(0, 1, 2, 3, 4, 5, 6))
    g.rhs_update(stage, 0.005)
    o.rhs(stage)
    o.update(stage, 0.005)
    same_fields(g, o, (0, 1, 2, 3, 4, 5))


VARIANTS = [(tb, ov) for tb in (True, False) for ov in (True, False)]


@pytest.fixture(params=["rw", "plain"])
def sweep(request, monkeypatch):
    """The implementations of the fused red-black sweep: the row-warp one fed
    by TMA (default for red-black-fast) and the plain-load one."""
    monkeypatch.setenv("LCS_B200_FUSED_SWEEP", request.param)
    return request.param


@pytest.mark.parametrize("tb,ov", VARIANTS)
@pytest.mark.parametrize("coloring,block", [(F.COLORING_RED_BLACK_FAST, 0), (F.COLORING_RED_BLACK, 0),
                                            (F.COLORING_RED_BLACK_BLOCK, 2)])
def test_hsmac_reference_setting_bitwise(tb, ov, coloring, block, sweep):
    """The reference's couple test: 16^3, h=3, omega 1.7, epsp 1e-3, itrmin = itrmax = 6,
    random haloed U, V, W, P (test/test_flows.jl:82-101)."""
    cfg = make_config(16, mode=F.MODE_FLOW, time_blocking=tb, overlap=ov, coloring=coloring, block=block)
    g, o = pair(cfg)
    load_random_flow([g, o], seed=10)
    lg = g.couple(2, 0.01)
    lo = o.couple(2, 0.01)
    assert lg["itr"] == lo["itr"] and lg["sweeps"] == lo["sweeps"]
    assert abs(lg["div"] - lo["div"]) <= 1e-12 * lo["div"]
    same_fields(g, o, (0, 1, 2, 6))


@pytest.mark.parametrize("tb,ov", VARIANTS)
@pytest.mark.parametrize("n,epsp", [(34, 2e-2), (64, 2e-2), (34, 1e3)])
def test_hsmac_long_runs_and_early_exit(tb, ov, n, epsp, sweep):
    """Partial tiles (n = 34), several z chunks (n = 64), a data-dependent exit,
    and an exit at exactly itrmin (epsp = 1e3)."""
    cfg = make_config(n, mode=F.MODE_FLOW, time_blocking=tb, overlap=ov, itrmin=6, itrmax=60, epsp=epsp)
    g, o = pair(cfg)
    stage = 1 if ov else 2  # couple! on Us2 in stage 1, on Us in stage 2
    fs = (3, 4, 5, 6) if stage == 1 else (0, 1, 2, 6)
    rng = np.random.default_rng(20 + n)
    for f in fs:
        a = rng.standard_normal(g.interior_shape) * 0.1
        g.field_set(f, a)
        o.field_set(f, a)
    lg = g.couple(stage, 0.004)
    lo = o.couple(stage, 0.004)
    assert lg["itr"] == lo["itr"] and lg["sweeps"] == lo["sweeps"]
    if epsp > 1:
        assert lg["itr"] == 6 and lg["sweeps"] == 7
    assert abs(lg["div"] - lo["div"]) <= 1e-12 * lo["div"]
    same_fields(g, o, fs)


@pytest.mark.parametrize("tb,ov", VARIANTS)
def test_row_warp_sweep_equals_plain_sweep_128(tb, ov, monkeypatch):
    """At 128^3 (several tiles and z chunks per sweep) the TMA-fed row-warp
    sweep and the plain-load sweep give identical fields."""
    from lcs_b200 import inits

    out = []
    for mode in ("rw", "plain"):
        monkeypatch.setenv("LCS_B200_FUSED_SWEEP", mode)
        e = Engine(make_config(128, mode=F.MODE_FLOW, time_blocking=tb, overlap=ov, itrmin=6, itrmax=12,
                               epsp=1e-12))
        U, V, W, P = inits.spectral_flow(128, seed=4)
        e.upload_flow(U, V, W, P)
        lg = e.couple(2, 0.003)
        out.append((lg, e.download_flow()))
        e.close()
    lb, fb = out[-1]
    for la, fa in out[:-1]:
        assert la["itr"] == lb["itr"] and abs(la["div"] - lb["div"]) <= 1e-13 * lb["div"]
        for a, b in zip(fa, fb):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("variant", ["8", "5"])
def test_row_warp_variants_equal_default(variant, monkeypatch):
    """The row-warp sweep's other tile heights and ring depths give the same
    fields as the default one (96^3: partial tiles in x and y)."""
    from lcs_b200 import inits

    out = []
    for v in (variant, "13"):
        monkeypatch.setenv("LCS_B200_RW", v)
        e = Engine(make_config(96, mode=F.MODE_FLOW, time_blocking=True, overlap=True, itrmin=6, itrmax=9,
                               epsp=1e-12))
        U, V, W, P = inits.spectral_flow(96, seed=11)
        e.upload_flow(U, V, W, P)
        lg = e.couple(2, 0.003)
        out.append((lg, e.download_flow()))
        e.close()
    (la, fa), (lb, fb) = out
    assert la["itr"] == lb["itr"] and abs(la["div"] - lb["div"]) <= 1e-13 * lb["div"]
    for a, b in zip(fa, fb):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("tb", [True, False])
@pytest.mark.parametrize("coloring", [F.COLORING_RED_BLACK_FAST, F.COLORING_RED_BLACK])
def test_face_kernel_equals_sequential_face_phases(tb, coloring, monkeypatch):
    """The overlap sweep's face slabs: the one cooperative launch (opposite
    faces together, grid barriers between phases) and the twelve in-place
    launches of the reference's order give identical fields and residuals."""
    from lcs_b200 import inits

    out = []
    for mode in ("coop", "phases"):
        monkeypatch.setenv("LCS_B200_FACES", mode)
        e = Engine(make_config(96, mode=F.MODE_FLOW, time_blocking=tb, overlap=True, coloring=coloring, itrmin=6,
                               itrmax=15, epsp=1e-12))
        U, V, W, P = inits.spectral_flow(96, seed=7)
        e.upload_flow(U, V, W, P)
        lg = e.couple(2, 0.003)
        out.append((lg, e.download_flow()))
        e.close()
    (la, fa), (lb, fb) = out
    # the residual is summed over differently grouped partials: equal to rounding
    assert la["itr"] == lb["itr"] and la["sweeps"] == lb["sweeps"]
    assert abs(la["div"] - lb["div"]) <= 1e-13 * lb["div"]
    for a, b in zip(fa, fb):
        assert np.array_equal(a, b)


def test_synchalo_bitwise():
    cfg = make_config(12, mode=F.MODE_FLOW)
    g, o = pair(cfg)
    load_random_flow([g, o], seed=5, fields=(0, 1, 2, 3, 4, 5, 6))
    for r, full in ((3, True), (1, True), (3, False), (2, False)):
        g.synchalo([0, 4, 6], r, full)
        o.synchalo([0, 4, 6], r, full)
        same_fields(g, o, (0, 4, 6), haloed=True)


def test_timestep_bitwise():
    cfg = make_config(24, Re=80.0, species=[{"n": 30, "density_ratio": 843.0}, {"n": 20, "density_ratio": 100.0}])
    g, o = pair(cfg)
    rng = np.random.default_rng(6)
    for f in (0, 1, 2):
        a = rng.standard_normal(g.interior_shape)
        g.field_set(f, a)
        o.field_set(f, a)
    load_particles([g, o], 0, 30, seed=1, diam=0.01)
    load_particles([g, o], 1, 20, seed=2, diam=0.03)
    assert g.flow_timestep() == o.flow_timestep()
    assert g.particles_timestep() == o.particles_timestep()
    assert g.timestep() == o.timestep()


@pytest.mark.parametrize("forcing", [F.FORCING_LINEAR_POWER, F.FORCING_RC_ENERGY])
@pytest.mark.parametrize("n,coarse,kmax", [(16, 4, 2), (32, 8, 2), (32, 8, 3), (64, 4, 2), (256, 16, 2)])
def test_forcing(forcing, n, coarse, kmax):
    """Both forcings on random fields; (64, 4) and (256, 16) give the 16-cell
    box filter of the rc256 workload (filter size n / coarse_size)."""
    cfg = make_config(n, mode=F.MODE_FLOW, forcing=forcing, power=0.5, energy=0.649, kmin=1, kmax=kmax,
                      coarse=coarse)
    g, o = pair(cfg)
    rng = np.random.default_rng(7)
    for f in (0, 1, 2):
        a = rng.standard_normal(g.interior_shape)
        g.field_set(f, a)
        o.field_set(f, a)
    pg = g.forcing(0.01)
    po = o.forcing(0.01)
    assert abs(pg["p"] - po["p"]) <= 1e-12 * abs(po["p"])
    if forcing == F.FORCING_RC_ENERGY:
        assert pg["e10"] == po["e10"] == 0.649
    for f in (0, 1, 2):
        assert rel_l2(g.field_get(f), o.field_get(f)) <= 1e-13


@pytest.mark.parametrize("drag", [F.DRAG_LINEAR, F.DRAG_NONLINEAR])
@pytest.mark.parametrize("stage", [1, 2])
def test_particles_bitwise(drag, stage):
    n, npart = 16, 1000
    cfg = make_config(n, Re=30.0, species=[{"n": npart, "density_ratio": 3.0, "gravity": 9.8, "drag": drag}])
    g, o = pair(cfg)
    load_random_flow([g, o], seed=8, fields=(0, 1, 2, 3, 4, 5))
    load_particles([g, o], 0, npart, seed=9, spread=1.3, diam=0.2)  # some particles outside [0, 2pi)
    for fn in ("boundary", "motion"):
        getattr(g, "particles_" + fn)(0, stage)
        getattr(o, "particles_" + fn)(0, stage)
    g.particles_update(0, stage, 0.003)
    o.particles_update(0, stage, 0.003)
    for p in range(F.NPROP):
        a, b = g.prop_get(0, p), o.prop_get(0, p)
        if drag == F.DRAG_NONLINEAR and p >= F.PROP_U:
            # pow(Rep, 0.687): CUDA's pow and glibc's may differ in the last bit
            assert np.allclose(a, b, rtol=1e-14, atol=0), F.PROP_NAMES[p]
        else:
            assert np.array_equal(a, b), F.PROP_NAMES[p]


def test_particle_mapping_indices_bitwise():
    """Mapping(i, j, k) of interp.jl:92-126 is integer work: compared exactly
    through an indicator field that encodes the cell index in the value."""
    n, npart = 32, 4096
    cfg = make_config(n, species=[{"n": npart}])
    g, o = pair(cfg)
    hshape = g.haloed_shape
    code = np.arange(np.prod(hshape), dtype=np.float64).reshape(hshape)
    for e in (g, o):
        e.field_set(0, code, haloed=True)
        e.field_set(1, code, haloed=True)
        e.field_set(2, code, haloed=True)
    rng = np.random.default_rng(4)
    L = 2 * math.pi
    x, y, z = (rng.random(npart) * L for _ in range(3))
    # place particles exactly on nodes: weights (1,0) make interp return the code of (i, j, k)
    dx = L / n
    xi, yi, zi = (np.floor(a / dx) * dx for a in (x, y, z))
    zero = np.zeros(npart)
    for e in (g, o):
        e.upload_particles(0, np.ones(npart), xi, yi, zi, zero, zero, zero)
    gv = [g.prop_get(0, p) for p in (F.PROP_X, F.PROP_Y, F.PROP_Z)]
    ov = [o.prop_get(0, p) for p in (F.PROP_X, F.PROP_Y, F.PROP_Z)]
    for a, b in zip(gv, ov):
        assert np.array_equal(a, b)
    g.particles_motion(0, 1)
    o.particles_motion(0, 1)
    assert np.array_equal(g.prop_get(0, F.PROP_DUDT), o.prop_get(0, F.PROP_DUDT))


def test_init_particle_velocity_bitwise():
    cfg = make_config(32, species=[{"n": 5000}])
    g, o = pair(cfg)
    load_random_flow([g, o], seed=11, fields=(0, 1, 2), haloed=False)
    load_particles([g, o], 0, 5000, seed=12)
    g.init_particle_velocity(0)
    o.init_particle_velocity(0)
    for p in (F.PROP_U, F.PROP_V, F.PROP_W):
        assert np.array_equal(g.prop_get(0, p), o.prop_get(0, p))


def evolve_pair(cfg, steps, seed=0, nparts=(2000,), graphs=False):
    from lcs_b200 import inits

    n = cfg.dims[0]
    engines = pair(cfg)
    U, V, W, P = inits.spectral_flow(n, seed=seed)
    for e in engines:
        e.upload_flow(U, V, W, P)
    for s, npart in enumerate(nparts):
        x, y, z = inits.random_positions(npart, seed + 7 + s)
        zero = np.zeros(npart)
        diam = np.full(npart, 0.02 * (s + 1))
        for e in engines:
            e.upload_particles(s, diam, x, y, z, zero, zero, zero)
            e.init_particle_velocity(s)
    logs = []
    for e in engines:
        if graphs and isinstance(e, Engine) and not isinstance(e, OracleEngine):
            logs.append(e.step(steps))
        else:
            lg = []
            for _ in range(steps):
                dt = e.timestep()
                lg.append(e.evolve(dt))
            logs.append(lg)
    return engines, logs


@pytest.mark.parametrize("forcing", [F.FORCING_LINEAR_POWER, F.FORCING_RC_ENERGY])
@pytest.mark.parametrize("graphs", [False, True])
def test_ten_steps_rel_l2(forcing, graphs, sweep):
    """North-star parity: fields rel-L2 <= 1e-10 after 10 steps (config-0 style)."""
    cfg = make_config(32, forcing=forcing, power=0.5, energy=0.649, kmin=1, kmax=2, coarse=8, Re=100.0,
                      itrmin=6, itrmax=40, epsp=1e-8 * 2 * math.pi / 32, graphs=int(graphs),
                      species=[{"n": 2000, "density_ratio": 843.0}, {"n": 1000, "density_ratio": 843.0}])
    (g, o), (lg, lo) = evolve_pair(cfg, 10, nparts=(2000, 1000), graphs=graphs)
    for a, b in zip(lg, lo):
        assert a["couple1"]["itr"] == b["couple1"]["itr"] and a["couple2"]["itr"] == b["couple2"]["itr"]
        assert abs(a["dt"] - b["dt"]) <= 1e-13 * b["dt"]
    fg, fo = g.download_flow(), o.download_flow()
    for a, b in zip(fg, fo):
        assert rel_l2(a, b) <= 1e-10
    for s in (0, 1):
        pg, po = g.download_particles(s), o.download_particles(s)
        for k in ("x", "y", "z", "u", "v", "w"):
            assert rel_l2(pg[k], po[k]) <= 1e-10
    assert g.get_state()[0] == o.get_state()[0] == 10


def test_graph_step_equals_direct_calls():
    """lcs_step (device-resident CUDA graph with WHILE-node couples) is the
    same computation as timestep!/evolve! issued call by call."""
    base = dict(forcing=F.FORCING_LINEAR_POWER, power=0.5, Re=100.0, itrmin=6, itrmax=30, epsp=1e-7,
                species=[{"n": 3000, "density_ratio": 843.0}])
    from lcs_b200 import inits

    res = []
    for graphs in (0, 1):
        e = Engine(make_config(48, graphs=graphs, **base))
        U, V, W, P = inits.spectral_flow(48, seed=3)
        e.upload_flow(U, V, W, P)
        x, y, z = inits.random_positions(3000, 5)
        zero = np.zeros(3000)
        e.upload_particles(0, np.full(3000, 0.02), x, y, z, zero, zero, zero)
        e.init_particle_velocity(0)
        logs = e.step(5)
        res.append((e.download_flow(), e.download_particles(0), logs))
    (fa, pa, la), (fb, pb, lb) = res
    for a, b in zip(fa, fb):
        assert np.array_equal(a, b)
    for k in ("x", "u"):
        assert np.array_equal(pa[k], pb[k])
    assert [x["couple2"]["itr"] for x in la] == [x["couple2"]["itr"] for x in lb]


def test_empty_species_rejected_and_flow_mode():
    """An empty species makes the reference's `maximum(diams)` throw; both
    libraries refuse it at create time.  FlowMode (no particles) runs."""
    from lcs_b200 import LCSError

    bad = make_config(16, species=[{"n": 0}, {"n": 10}])
    for cls in (Engine, OracleEngine):
        with pytest.raises(LCSError) as ei:
            cls(bad)
        assert ei.value.code == F.EINVAL
    cfg = make_config(16, mode=F.MODE_FLOW, forcing=F.FORCING_NO, Re=50.0, itrmax=12)
    (g, o), _ = evolve_pair(cfg, 2, nparts=())
    for a, b in zip(g.download_flow(), o.download_flow()):
        assert rel_l2(a, b) <= 1e-12


def test_errors_are_reported_not_raised_across_the_abi():
    cfg = make_config(16)
    g = Engine(cfg)
    from lcs_b200 import LCSError

    with pytest.raises(LCSError) as ei:
        g.evolve(0.01)  # no flow uploaded yet
    assert ei.value.code == F.ESTATE
    with pytest.raises(LCSError):
        g.rhs(3)
    with pytest.raises(LCSError):
        g.prop_get(5, 0)


NONCUBIC = [(40, 24, 32), (70, 34, 96), (96, 40, 18)]


@pytest.mark.parametrize("tb,ov", VARIANTS)
@pytest.mark.parametrize("dims", NONCUBIC)
def test_hsmac_noncubic_bitwise(dims, tb, ov, sweep):
    """Grids with a different size per axis (per-axis spacings; several tile
    columns and rows, partial tiles, few z planes): the couple's fields are
    bit-identical to the oracle's, itr is equal and the residual agrees to
    1e-12."""
    cfg = make_config(dims=dims, mode=F.MODE_FLOW, time_blocking=tb, overlap=ov, itrmin=6, itrmax=20, epsp=1e-12,
                      Re=50.0)
    g, o = pair(cfg)
    rng = np.random.default_rng(sum(dims))
    for f in (0, 1, 2, 6):
        a = rng.standard_normal(g.interior_shape) * (0.1 if f == 6 else 0.5)
        g.field_set(f, a)
        o.field_set(f, a)
    lg = g.couple(2, 0.004)
    lo = o.couple(2, 0.004)
    assert lg["itr"] == lo["itr"] and lg["sweeps"] == lo["sweeps"]
    assert abs(lg["div"] - lo["div"]) <= 1e-12 * lo["div"]
    same_fields(g, o, (0, 1, 2, 6))


@pytest.mark.parametrize("graphs", [False, True])
def test_ten_steps_noncubic_rel_l2(graphs):
    """Ten full steps (linear-power forcing, two particle species) on a 48 x 32 x 40
    grid: couple itr equal, dt to 1e-13, fields and particles to rel-L2 <= 1e-10."""
    from lcs_b200 import inits

    dims = (48, 32, 40)
    cfg = make_config(dims=dims, forcing=F.FORCING_LINEAR_POWER, power=0.5, Re=100.0, itrmin=6, itrmax=40,
                      epsp=1e-8 * 2 * math.pi / 48, graphs=int(graphs),
                      species=[{"n": 2000, "density_ratio": 843.0}, {"n": 1000, "density_ratio": 843.0}])
    g, o = pair(cfg)
    rng = np.random.default_rng(5)
    for f in (0, 1, 2):
        a = rng.standard_normal(g.interior_shape) * 0.5
        g.field_set(f, a)
        o.field_set(f, a)
    for s, npart in enumerate((2000, 1000)):
        x, y, z = inits.random_positions(npart, 30 + s)
        zero = np.zeros(npart)
        for e in (g, o):
            e.upload_particles(s, np.full(npart, 0.02 * (s + 1)), x, y, z, zero, zero, zero)
            e.init_particle_velocity(s)
    lo = []
    for _ in range(10):
        lo.append(o.evolve(o.timestep()))
    if graphs:
        lg = g.step(10)
    else:
        lg = [g.evolve(g.timestep()) for _ in range(10)]
    for a, b in zip(lg, lo):
        assert a["couple1"]["itr"] == b["couple1"]["itr"] and a["couple2"]["itr"] == b["couple2"]["itr"]
        assert abs(a["dt"] - b["dt"]) <= 1e-13 * b["dt"]
    for a, b in zip(g.download_flow(), o.download_flow()):
        assert rel_l2(a, b) <= 1e-10
    for s in (0, 1):
        pg, po = g.download_particles(s), o.download_particles(s)
        for k in ("x", "y", "z", "u", "v", "w"):
            assert rel_l2(pg[k], po[k]) <= 1e-10
