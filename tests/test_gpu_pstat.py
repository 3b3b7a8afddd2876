"""Particle statistics on the device against the oracle (`Particles.stat`,
src/particles/stat.jl:113-151 with rdf.jl:1-103 and spectrum.jl:11-78;
`Particles.density`, stat.jl:176-215), in both precision forms (particle state
is FP64 in both).

Exact: pair counts, contact pairs, bin edges, g(r) (with dyadic diameters the
mean diameter is exact in any summation order), the SPH densities (same
accumulation order, no contracted multiply-adds) and the reordered species.
Summary means to 1e-12 relative (tree vs sequential sums); the spectrum to
1e-9 of its shot-noise scale 4 pi k^2 / N (the reference adds it with atomics,
in no fixed order)."""

import math

import numpy as np
import pytest

from helpers import make_config
from lcs_b200 import Engine, _abi
from oracle_engine import OracleEngine

pytestmark = pytest.mark.gpu
L = 2 * math.pi
PRECISIONS = [_abi.PRECISION_FP64, _abi.PRECISION_FP32_MIXED]


def pair(n, npart, seed, precision, dyadic_diam=None):
    cfg = make_config(dims=n, species=[{"n": npart, "density_ratio": 843.0}], Re=200.0, precision=precision)
    g, o = Engine(cfg), OracleEngine(cfg)
    rng = np.random.default_rng(seed)
    x, y, z = (rng.random(npart) * L for _ in range(3))
    u, v, w = (rng.standard_normal(npart) for _ in range(3))
    d = np.full(npart, dyadic_diam) if dyadic_diam else rng.random(npart) * 0.02 + 0.01
    for e in (g, o):
        e.upload_particles(0, d, x, y, z, u, v, w, ids=np.arange(1, npart + 1))
    return g, o


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("n,npart,ratio,ncell", [((32, 32, 32), 20000, 4, 2), ((48, 32, 40), 30000, 2, 1),
                                                 ((16, 16, 16), 5000, 1, 3)])
def test_particle_stat_equals_oracle(n, npart, ratio, ncell, precision):
    kw = dict(grid_ratio=ratio, bin_size=16, search_cell_size=ncell, contact_tolerance=0.9, min_radius=1e-3,
              max_wavenumber=32, nsamples=16)
    g, o = pair(n, npart, npart + ratio, precision, dyadic_diam=2.0 ** -6)
    a, b = g.particles_stat(0, 0.25, **kw), o.particles_stat(0, 0.25, **kw)
    for k in ("x", "y", "z", "u", "v", "w", "diam"):
        assert math.isclose(a[k]["mean"], b[k]["mean"], rel_tol=1e-12, abs_tol=1e-15), k
        assert a[k]["max"] == b[k]["max"] and a[k]["min"] == b[k]["min"], k
    assert a["taup"] == b["taup"] and a["St"] == b["St"]
    ra, rb = a["rdf"], b["rdf"]
    assert np.array_equal(ra["edges"], rb["edges"])
    assert np.array_equal(ra["npairs"], rb["npairs"]) and ra["npairs"].sum() > 0
    assert ra["npairs_contact"] == rb["npairs_contact"]
    assert np.array_equal(ra["gr"], rb["gr"]) and ra["gr_contact"] == rb["gr_contact"]
    sa, sb = a["spectrum"], b["spectrum"]
    assert np.array_equal(sa["wavenumbers"], sb["wavenumbers"])
    scale = 4 * math.pi * sa["wavenumbers"] ** 2 / npart
    assert np.all(np.abs(sa["Enp"] - sb["Enp"]) <= 1e-9 * scale), (sa["Enp"], sb["Enp"])
    # the species was reordered the same way
    pa, pb = g.download_particles(0), o.download_particles(0)
    for k in ("ids", "x", "y", "z", "u", "v", "w", "diam"):
        assert np.array_equal(pa[k], pb[k]), k
    g.close()
    o.close()


@pytest.mark.parametrize("precision", PRECISIONS)
def test_particle_stat_random_diameters(precision):
    """Random diameters: the mean differs in the last bits between orders, the
    pair counts per bin do not depend on it."""
    g, o = pair((32, 32, 32), 20000, 4, precision)
    kw = dict(grid_ratio=2, bin_size=32, search_cell_size=2, contact_tolerance=1e-3, min_radius=1e-3,
              max_wavenumber=8, nsamples=8)
    a, b = g.particles_stat(0, 0.5, **kw), o.particles_stat(0, 0.5, **kw)
    assert np.array_equal(a["rdf"]["npairs"], b["rdf"]["npairs"])
    assert math.isclose(a["taup"], b["taup"], rel_tol=1e-12)
    assert np.allclose(a["rdf"]["gr"], b["rdf"]["gr"], rtol=1e-15, atol=0)
    g.close()
    o.close()


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("n,npart,ratio", [((32, 32, 32), 30000, 2), ((24, 24, 24), 8000, 1)])
def test_density_equals_oracle(n, npart, ratio, precision):
    g, o = pair(n, npart, 7 * ratio, precision)
    ra, rb = g.particles_density(0, ratio), o.particles_density(0, ratio)
    assert np.array_equal(ra, rb)
    assert np.array_equal(g.download_particles(0)["ids"], o.download_particles(0)["ids"])
    g.close()
    o.close()


def test_particle_stat_large():
    """2^21 particles, 256^3 grid, the production settings (grid_ratio 4,
    16 bins, search 2 cells, 64 directions to k = 128): runs, and its counts
    agree with the counts of the same index recomputed from the downloaded
    state (total pairs, self-consistency of g(r))."""
    n, npart = (256, 256, 256), 1 << 21
    cfg = make_config(dims=n, species=[{"n": npart, "density_ratio": 843.0}], Re=200.0)
    g = Engine(cfg)
    rng = np.random.default_rng(1)
    x, y, z = (rng.random(npart) * L for _ in range(3))
    zero = np.zeros(npart)
    g.upload_particles(0, np.full(npart, 2.0 ** -8), x, y, z, zero, zero, zero, ids=np.arange(1, npart + 1))
    st = g.particles_stat(0, 1.0)
    r = st["rdf"]
    rho0 = (npart * (npart - 1) // 2) / L ** 3
    e = r["edges"]
    shell = (4.0 / 3.0) * math.pi * (e[1:] ** 3 - e[:-1] ** 3)
    assert np.allclose(r["gr"], r["npairs"] / shell / rho0, rtol=1e-14, atol=0)
    # uniform random particles: g(r) ~ 1 in the well-populated outer bins
    assert np.all(np.abs(r["gr"][-4:] - 1.0) < 0.05), r["gr"]
    # 14 shells up to k = 128 (the box itself gives the low shells their
    # weight: non-integer wave vectors are not orthogonal to the constant)
    assert st["spectrum"]["Enp"].size == 14 and np.all(np.isfinite(st["spectrum"]["Enp"]))
    g.close()
