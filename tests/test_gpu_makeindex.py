"""`Particles.makeindex!` (src/particles/makeindex.jl:29-67) on the device
against the oracle: hashes, starts, stops, the permuted properties and ids are
bit-exact for identical positions (integer and index work), in both precision
forms (particle state is FP64 in both).  At a large size the index is checked
through its own invariants (sortedness, the count invariant of
test/test_particles.jl:85, starts/stops against searchsorted)."""

import math

import numpy as np
import pytest

from helpers import make_config
from lcs_b200 import Engine, _abi
from oracle_engine import OracleEngine
from test_makeindex import cell_hash, out_of_domain_positions

pytestmark = pytest.mark.gpu
L = 2 * math.pi


def load(engines, npart, seed, positions=None):
    rng = np.random.default_rng(seed)
    if positions is None:
        positions = [rng.random(npart) * L for _ in range(3)]
    u, v, w = (rng.standard_normal(npart) for _ in range(3))
    diam = rng.random(npart)
    props = {p: rng.random(npart) * L for p in (_abi.PROP_X2, _abi.PROP_Y2, _abi.PROP_Z2, _abi.PROP_U2, _abi.PROP_V2,
                                                 _abi.PROP_W2, _abi.PROP_DUDT, _abi.PROP_DVDT, _abi.PROP_DWDT)}
    for e in engines:
        e.upload_particles(0, diam, *positions, u, v, w, ids=np.arange(1, npart + 1))
        for p, a in props.items():
            e.prop_set(0, p, a)


def same_index(g, o, ratio):
    for a, b in zip(g.particles_cellindex(0, ratio), o.particles_cellindex(0, ratio)):
        assert np.array_equal(a, b)
    for p in range(_abi.NPROP):
        assert np.array_equal(g.prop_get(0, p), o.prop_get(0, p)), p
    assert np.array_equal(g.download_particles(0)["ids"], o.download_particles(0)["ids"])


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_FP32_MIXED])
@pytest.mark.parametrize("n,ratio,npart,stage", [((16, 16, 16), 4, 10, 1), ((16, 16, 16), 1, 3000, 2),
                                                 ((24, 16, 20), 2, 20000, 1), ((64, 64, 64), 2, 300000, 2)])
def test_makeindex_equals_oracle(n, ratio, npart, stage, precision):
    cfg = make_config(dims=n, species=[{"n": npart, "density_ratio": 843.0}], precision=precision)
    g, o = Engine(cfg), OracleEngine(cfg)
    load((g, o), npart, npart + ratio)
    for e in (g, o):
        e.particles_makeindex(0, stage, ratio)
    same_index(g, o, ratio)
    # a second index over the sorted order (the reallocation-free path) is idempotent
    for e in (g, o):
        e.particles_makeindex(0, stage, ratio)
    same_index(g, o, ratio)
    g.close()
    o.close()


def test_makeindex_boundaries_and_ratio_change():
    """Positions on cell faces with many ties, then a different grid_ratio on
    the same handle (the index buffers are rebuilt)."""
    n, npart = (32, 32, 32), 5000
    rng = np.random.default_rng(11)
    dxc = (L / 32) * 4
    pos = [rng.integers(0, 8, npart) * dxc, np.where(rng.random(npart) < 0.5, 0.0, rng.integers(0, 8, npart) * dxc),
           rng.random(npart) * L]
    cfg = make_config(dims=n, species=[{"n": npart, "density_ratio": 843.0}])
    g, o = Engine(cfg), OracleEngine(cfg)
    load((g, o), npart, 11, positions=pos)
    for ratio in (4, 1, 8):
        for e in (g, o):
            e.particles_makeindex(0, 1, ratio)
        same_index(g, o, ratio)
    g.close()
    o.close()


def test_step_after_makeindex_equals_sorted_upload():
    """makeindex only reorders the particles: stepping after it equals stepping
    a handle whose particles were uploaded in the sorted order (bitwise)."""
    n, npart, ratio = 32, 4000, 2
    cfg = make_config(n, species=[{"n": npart, "density_ratio": 843.0}], Re=100.0)
    cfg.use_graphs = 1
    a, b = Engine(cfg), Engine(cfg)
    rng = np.random.default_rng(5)
    flow = [rng.standard_normal((n, n, n)) * 0.2 for _ in range(3)] + [np.zeros((n, n, n))]
    pos = [rng.random(npart) * L for _ in range(3)]
    zero = np.zeros(npart)
    diam = np.full(npart, 0.01)
    a.upload_flow(*flow)
    a.upload_particles(0, diam, *pos, zero, zero, zero, ids=np.arange(1, npart + 1))
    a.init_particle_velocity(0)
    a.particles_makeindex(0, 1, ratio)
    s = a.download_particles(0)
    perm = s["ids"] - 1
    b.upload_flow(*flow)
    b.upload_particles(0, diam, *(p[perm] for p in pos), zero, zero, zero, ids=s["ids"])
    b.init_particle_velocity(0)
    la, lb = a.step(3), b.step(3)
    assert [x["dt"] for x in la] == [x["dt"] for x in lb]
    pa, pb = a.download_particles(0), b.download_particles(0)
    for k in ("ids", "x", "y", "z", "u", "v", "w"):
        assert np.array_equal(pa[k], pb[k]), k
    for x, y in zip(a.download_flow(), b.download_flow()):
        assert np.array_equal(x, y)
    a.close()
    b.close()


def test_graph_steps_across_makeindex():
    """Graphs captured before an index keep stepping the moved species: steps,
    index, steps equals steps, the same reordering uploaded, steps (bitwise)."""
    n, npart, ratio = 32, 3000, 4
    cfg = make_config(n, species=[{"n": npart, "density_ratio": 843.0}, {"n": 700, "density_ratio": 100.0}], Re=100.0)
    cfg.use_graphs = 1
    a, b = Engine(cfg), Engine(cfg)
    rng = np.random.default_rng(9)
    flow = [rng.standard_normal((n, n, n)) * 0.2 for _ in range(3)] + [np.zeros((n, n, n))]
    for e in (a, b):
        e.upload_flow(*flow)
    for s, m in enumerate((npart, 700)):
        pos = [rng.random(m) * L for _ in range(3)]
        zero = np.zeros(m)
        for e in (a, b):
            e.upload_particles(s, np.full(m, 0.01 * (s + 1)), *pos, zero, zero, zero, ids=np.arange(1, m + 1))
            e.init_particle_velocity(s)
    a.step(2)
    b.step(2)
    a.particles_makeindex(0, 1, ratio)
    perm = a.download_particles(0)["ids"] - 1
    props = {p: b.prop_get(0, p)[perm] for p in range(_abi.NPROP)}
    ids = b.download_particles(0)["ids"][perm]
    for p, v in props.items():
        b.prop_set(0, p, v)
    d = props[_abi.PROP_DIAM]
    b.upload_particles(0, d, props[_abi.PROP_X], props[_abi.PROP_Y], props[_abi.PROP_Z], props[_abi.PROP_U],
                       props[_abi.PROP_V], props[_abi.PROP_W], ids=ids)
    la, lb = a.step(3), b.step(3)
    assert [x["dt"] for x in la] == [x["dt"] for x in lb]
    for s in (0, 1):
        pa, pb = a.download_particles(s), b.download_particles(s)
        for k in ("ids", "x", "y", "z", "u", "v", "w"):
            assert np.array_equal(pa[k], pb[k]), (s, k)
        for p in range(_abi.NPROP):
            assert np.array_equal(a.prop_get(s, p), b.prop_get(s, p)), (s, p)
    a.close()
    b.close()


def test_makeindex_large_invariants():
    """2^22 particles in 256^3 cells of ratio 2: the index against its own
    invariants and the restated hash of the downloaded positions."""
    n, ratio, npart = (256, 256, 256), 2, 1 << 22
    cfg = make_config(dims=n, species=[{"n": npart, "density_ratio": 843.0}])
    g = Engine(cfg)
    rng = np.random.default_rng(2)
    pos = [rng.random(npart) * L for _ in range(3)]
    zero = np.zeros(npart)
    g.upload_particles(0, np.ones(npart), *pos, zero, zero, zero, ids=np.arange(1, npart + 1))
    g.particles_makeindex(0, 1, ratio)
    hashes, starts, stops = g.particles_cellindex(0, ratio)
    s = g.download_particles(0)
    assert int(np.sum(stops - starts + 1)) == npart
    assert np.all(np.diff(hashes) >= 0)
    assert np.array_equal(hashes, cell_hash(s["x"], s["y"], s["z"], n, ratio))
    perm = s["ids"] - 1
    assert np.array_equal(np.sort(perm), np.arange(npart))
    assert np.array_equal(s["x"], pos[0][perm])
    # stable: ids ascending inside every run of equal hashes
    same = hashes[1:] == hashes[:-1]
    assert np.all(s["ids"][1:][same] > s["ids"][:-1][same])
    xs = np.arange(1, starts.size + 1)
    assert np.array_equal(starts, np.searchsorted(hashes, xs, side="left") + 1)
    assert np.array_equal(stops, np.searchsorted(hashes, xs, side="right"))
    g.close()


def test_makeindex_outside_the_domain():
    """Positions just outside [0, 2pi) (halo cells 0 and nc+1): the same hashes,
    order and properties as the oracle."""
    n, npart = (32, 32, 32), 20000
    cfg = make_config(dims=n, species=[{"n": npart, "density_ratio": 843.0}])
    g, o = Engine(cfg), OracleEngine(cfg)
    load((g, o), npart, 12, positions=out_of_domain_positions(npart, 12))
    for ratio in (4, 1):
        for e in (g, o):
            e.particles_makeindex(0, 1, ratio)
        same_index(g, o, ratio)
    g.close()
    o.close()
