"""Particle statistics on the oracle (`Particles.stat`, src/particles/stat.jl:
113-151; rdf_assume_ci, src/particles/rdf.jl:1-103; spectrum,
src/particles/spectrum.jl:11-78; density, stat.jl:176-215) against
independent numpy restatements: brute-force pair loops over all particle pairs
restricted to the reference's cell neighbourhoods, and vectorised sums.

The reference's golden values for these (test/references/particles.jld2) are
git-LFS stubs; its rdf/density tests run on 10 particles in [0, 1)^3 with
Cell(4) and RDF(1e-3, 4, 1e-2, 1) (test/test_particles.jl:17-31, 160-182),
which test_reference_setup_runs repeats with seeded inputs.
"""

import math

import numpy as np
import pytest

from helpers import make_config
from lcs_b200 import _abi
from oracle_engine import OracleEngine

L = 2 * math.pi
WAVENUMBERS = (1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512, 768)


def setup(n, npart, seed, lo=0.0, hi=L, diam=None, ids=None):
    cfg = make_config(dims=n, species=[{"n": npart, "density_ratio": 843.0}], Re=200.0)
    e = OracleEngine(cfg)
    rng = np.random.default_rng(seed)
    x, y, z = (lo + rng.random(npart) * (hi - lo) for _ in range(3))
    u, v, w = (rng.standard_normal(npart) for _ in range(3))
    d = rng.random(npart) * 0.02 + 0.01 if diam is None else np.full(npart, diam)
    e.upload_particles(0, d, x, y, z, u, v, w, ids=np.arange(1, npart + 1) if ids is None else ids)
    return e, dict(x=x, y=y, z=z, u=u, v=v, w=w, diam=d)


def cells(x, y, z, n, ratio):
    return [np.floor(c / ((L / n[a]) * ratio)).astype(np.int64) + 1 for a, c in enumerate((x, y, z))]


def brute_rdf(st, P, ids, n, ratio, ncell, tol):
    """All pairs id1 < id2 whose cells differ by <= ncell on every axis (the
    first particle in a domain cell), binned by searchsortedfirst(edges, d) - 1."""
    x, y, z = P["x"], P["y"], P["z"]
    nc = [d // ratio for d in n]
    c = cells(x, y, z, n, ratio)
    edges = st["rdf"]["edges"]
    nb = len(edges) - 1
    dm = st["diam"]["mean"]
    counts = np.zeros(nb, np.int64)
    contact = 0
    for i in range(x.size):
        if not all(1 <= c[a][i] <= nc[a] for a in range(3)):
            continue
        near = np.ones(x.size, bool)
        for a in range(3):
            near &= np.abs(c[a] - c[a][i]) <= ncell
        near &= ids[i] < ids
        j = np.nonzero(near)[0]
        dx, dy, dz = x[i] - x[j], y[i] - y[j], z[i] - z[j]
        d = np.sqrt(dx * dx + dy * dy + dz * dz)
        k = np.searchsorted(edges, d, side="left")  # searchsortedfirst - 1
        ok = (k >= 1) & (k <= nb)
        np.add.at(counts, k[ok] - 1, 1)
        contact += int(np.sum(np.abs(d / dm - 1.0) < tol))
    return counts, contact


@pytest.mark.parametrize("n,npart,ratio,ncell", [((32, 32, 32), 3000, 4, 2), ((24, 16, 32), 2000, 2, 1),
                                                 ((16, 16, 16), 1500, 1, 3)])
def test_particle_stat_against_numpy(n, npart, ratio, ncell):
    e, P = setup(n, npart, 3 + ratio)
    tau_eta = 0.37
    st = e.particles_stat(0, tau_eta, grid_ratio=ratio, bin_size=16, search_cell_size=ncell, contact_tolerance=0.5,
                          min_radius=1e-3, max_wavenumber=16, nsamples=12)
    for k in ("x", "y", "z", "u", "v", "w", "diam"):
        a = P[k]
        assert math.isclose(st[k]["mean"], float(np.mean(a)), rel_tol=1e-12, abs_tol=1e-15)
        assert st[k]["max"] == a.max() and st[k]["min"] == a.min()
    dm = st["diam"]["mean"]
    Re = 200.0
    assert st["taup"] == 1.0 / 18.0 * 843.0 * Re * (dm * dm)
    assert st["St"] == st["taup"] / tau_eta
    # edges: logrange(min_radius, search_cell_size * dx, 17), endpoints exact
    edges = st["rdf"]["edges"]
    rmax = ncell * min(L / d for d in n)
    assert edges[0] == 1e-3 and edges[-1] == rmax
    assert np.allclose(edges, np.geomspace(1e-3, rmax, 17), rtol=1e-15, atol=0)
    # pair counts: the particle order changed (makeindex!), the pairs did not
    s = e.download_particles(0)
    S = dict(x=s["x"], y=s["y"], z=s["z"])
    counts, contact = brute_rdf(st, S, s["ids"], n, ratio, ncell, 0.5)
    assert np.array_equal(st["rdf"]["npairs"], counts)
    assert st["rdf"]["npairs_contact"] == contact
    rho0 = (npart * (npart - 1) // 2) / (L * L * L)
    shell = (4.0 / 3.0) * math.pi * (edges[1:] ** 3 - edges[:-1] ** 3)
    assert np.allclose(st["rdf"]["gr"], counts / shell / rho0, rtol=1e-14, atol=0)
    # spectrum: Fibonacci directions, vectorised sums
    ns = 12
    i = np.arange(ns)
    y = 1 - (i / (ns - 1)) * 2
    rad = np.sqrt(1 - y * y)
    th = math.pi * (3 - math.sqrt(5)) * i
    dirs = np.stack([np.cos(th) * rad, y, np.sin(th) * rad], 1)
    nsh = sum(1 for k in WAVENUMBERS if k <= 16)
    assert list(st["spectrum"]["wavenumbers"]) == list(WAVENUMBERS[:nsh])
    X = np.stack([S["x"], S["y"], S["z"]], 1)
    for b in range(nsh):
        kk = WAVENUMBERS[b]
        kd = X @ (kk * dirs).T
        cs, sn = np.cos(kd).sum(0), np.sin(kd).sum(0)
        enp = np.sum((cs ** 2 + sn ** 2) / npart ** 2 - 1 / npart) / ns * 4 * math.pi * kk ** 2
        scale = 4 * math.pi * kk ** 2 / npart  # the size of the shot-noise term
        assert abs(st["spectrum"]["Enp"][b] - enp) <= 1e-9 * scale, (b, st["spectrum"]["Enp"][b], enp)
    e.close()


def test_density_against_numpy():
    n, npart, ratio = (32, 32, 32), 3000, 2
    e, P = setup(n, npart, 9)
    rho = e.particles_density(0, ratio)
    s = e.download_particles(0)
    x, y, z = s["x"], s["y"], s["z"]
    h = min(L / d for d in n)
    c = cells(x, y, z, n, ratio)
    factor = 1 / (math.pi * h ** 3)
    ref = np.zeros(npart)
    for i in range(npart):
        near = np.ones(npart, bool)
        for a in range(3):
            near &= np.abs(c[a] - c[a][i]) <= 1
        j = np.nonzero(near)[0]
        d = np.sqrt((x[i] - x[j]) ** 2 + (y[i] - y[j]) ** 2 + (z[i] - z[j]) ** 2)
        d = d[d < 2 * h]
        q = d / h
        w = np.where(q < 1, factor * (1 - 1.5 * q ** 2 + 0.75 * q ** 3), factor * 0.25 * (2 - q) ** 3)
        ref[i] = w.sum()
    assert np.allclose(rho, ref, rtol=1e-12, atol=0)
    assert np.all(rho >= factor * 1.0 - 1e-12)  # every particle counts itself (d = 0)
    e.close()


def test_reference_setup_runs():
    """test_particles.jl:160-182 with seeded inputs: 10 particles in [0, 1)^3,
    16^3 grid, Cell(4), RDF(1e-3, 4, 1e-2, 1), diam 1, Spectrum(8, 8)."""
    e, P = setup((16, 16, 16), 10, 0, lo=0.0, hi=1.0, diam=1.0)
    st = e.particles_stat(0, 1.0, grid_ratio=4, bin_size=4, search_cell_size=1, contact_tolerance=1e-3,
                          min_radius=1e-2, max_wavenumber=8, nsamples=8)
    assert st["rdf"]["edges"].size == 5 and st["spectrum"]["Enp"].size == 6
    assert st["rdf"]["npairs"].sum() <= 45
    rho = e.particles_density(0, 4)
    assert rho.shape == (10,) and np.all(rho > 0)
    e.close()


def test_stat_errors():
    e, _ = setup((16, 16, 16), 10, 0)
    for kw in ({"bin_size": 0}, {"bin_size": 2000}, {"nsamples": 1}, {"min_radius": 0.0}, {"grid_ratio": 3}):
        with pytest.raises(Exception) as exc:
            e.particles_stat(0, 1.0, **kw)
        assert getattr(exc.value, "code", None) == _abi.EINVAL
    e.close()
