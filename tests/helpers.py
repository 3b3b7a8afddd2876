"""Config builders and seeded inputs shared by the tests."""

import math

import numpy as np

from lcs_b200 import _abi


def make_config(n=16, *, mode=_abi.MODE_FLOW_PARTICLE, h=3, time_blocking=True, overlap=True,
                coloring=_abi.COLORING_RED_BLACK_FAST, block=0, omega=1.7, epsp=1e-3, itrmin=6, itrmax=6,
                forcing=_abi.FORCING_NO, power=1.0, energy=1.0, kmin=1, kmax=2, coarse=4, Re=1.0,
                species=(), cfl=0.3, dtmax=0.01, graphs=0, dims=None, precision=_abi.PRECISION_FP64):
    """An lcs_config; defaults follow the reference's unit tests (test/test_flows.jl:11-21,
    FlowParams(1,1,1), HSMAC(.., RedBlackFast, 1.7, 1e-3, 6, 6))."""
    c = _abi.Config()
    c.abi_version = _abi.ABI_VERSION
    c.mode = mode
    d = dims or (n, n, n)
    for a in range(3):
        c.dims[a] = d[a]
    c.halo_size = h
    c.cfl, c.dtmax = cfl, dtmax
    c.U0, c.L0, c.NU = 1.0, 1.0, 1.0 / Re
    c.time_blocking, c.overlap, c.coloring, c.coloring_block = int(time_blocking), int(overlap), coloring, block
    c.omega, c.epsp, c.itrmin, c.itrmax = omega, epsp, itrmin, itrmax
    c.forcing, c.power, c.energy = forcing, power, energy
    c.kmin, c.kmax, c.coarse_size = kmin, kmax, coarse
    c.n_species = len(species)
    for s, sp in enumerate(species):
        c.species[s].nvalid = sp.get("n", 10)
        c.species[s].gravity = sp.get("gravity", 0.0)
        c.species[s].density_ratio = sp.get("density_ratio", 1.0)
        c.species[s].drag = sp.get("drag", _abi.DRAG_LINEAR)
    c.precision = precision
    c.device = 0
    c.use_graphs = graphs
    return c


def rand_haloed(eng, rng):
    """Random values on the whole haloed box (the reference's rand!.(fields.Us))."""
    return rng.random(eng.haloed_shape)


def rand_interior(eng, rng):
    return rng.random(eng.interior_shape)


def load_random_flow(engines, seed=0, haloed=True, fields=(0, 1, 2, 6)):
    """Same random haloed U, V, W, P into every engine; returns the arrays."""
    rng = np.random.default_rng(seed)
    out = {}
    for f in fields:
        a = rng.random(engines[0].haloed_shape if haloed else engines[0].interior_shape)
        out[f] = a
        for e in engines:
            e.field_set(f, a, haloed=haloed)
    return out


def load_particles(engines, species, n, seed=0, spread=1.0, diam=1.0):
    """Same random particle state (positions in [0, 2pi*spread)) into every engine."""
    rng = np.random.default_rng(seed + 101 * species)
    L = 2 * math.pi
    x, y, z = (rng.random(n) * L * spread for _ in range(3))
    u, v, w = (rng.random(n) for _ in range(3))
    d = np.full(n, diam)
    for e in engines:
        e.upload_particles(species, d, x, y, z, u, v, w, ids=np.arange(1, n + 1))
    props = {}
    for p in (_abi.PROP_X2, _abi.PROP_Y2, _abi.PROP_Z2, _abi.PROP_U2, _abi.PROP_V2, _abi.PROP_W2,
              _abi.PROP_DUDT, _abi.PROP_DVDT, _abi.PROP_DWDT):
        a = rng.random(n) * (L if p <= _abi.PROP_Z2 else 1.0)
        props[p] = a
        for e in engines:
            e.prop_set(species, p, a)
    return props


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0)
