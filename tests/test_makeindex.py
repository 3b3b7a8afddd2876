"""`Particles.makeindex!` (src/particles/makeindex.jl:29-67) on the oracle.

The reference's golden arrays for this test (test/references/particles.jld2)
are git-LFS stubs, so the pin is its own assertion, sum(stops - starts + 1) ==
nvalid (test/test_particles.jl:85), on its own setup (a 16^3 grid, Cell(4),
10 random particles, test_particles.jl:17-31), plus properties any correct
index has: hashes sorted and equal to the restated cell hash of each sorted
particle, equal hashes in their original order (a stable sort), starts/stops
equal to numpy's searchsorted, every property permuted with the ids.
"""

import math

import numpy as np
import pytest

from helpers import make_config
from lcs_b200 import _abi
from oracle_engine import OracleEngine

L = 2 * math.pi


def cell_hash(x, y, z, n, ratio):
    """Restated hash of makeindex.jl:47-52 with hasher.jl:15-38 (1-based, axes 0:nc+1)."""
    nc = [d // ratio for d in n]
    h = np.ones(x.shape, np.int64)
    stride = 1
    for a, c in enumerate((x, y, z)):
        dxc = (L / n[a]) * ratio
        ci = np.floor((c - 0.0) / dxc).astype(np.int64) + 1
        h += ci * stride
        stride *= nc[a] + 2
    return h


def setup(n, npart, seed, ratio, positions=None):
    cfg = make_config(dims=n, species=[{"n": npart, "density_ratio": 843.0}])
    e = OracleEngine(cfg)
    rng = np.random.default_rng(seed)
    if positions is None:
        positions = [rng.random(npart) * L for _ in range(3)]
    x, y, z = positions
    u, v, w = (rng.standard_normal(npart) for _ in range(3))
    diam = rng.random(npart)
    e.upload_particles(0, diam, x, y, z, u, v, w, ids=np.arange(1, npart + 1))
    extra = {}
    for p in (_abi.PROP_X2, _abi.PROP_Y2, _abi.PROP_Z2, _abi.PROP_U2, _abi.PROP_V2, _abi.PROP_W2,
              _abi.PROP_DUDT, _abi.PROP_DVDT, _abi.PROP_DWDT):
        extra[p] = rng.random(npart) * L
        e.prop_set(0, p, extra[p])
    before = {p: e.prop_get(0, p) for p in range(_abi.NPROP)}
    return e, before


def check_index(e, before, n, ratio, stage):
    e.particles_makeindex(0, stage, ratio)
    hashes, starts, stops = e.particles_cellindex(0, ratio)
    npart = hashes.size
    nc = [d // ratio for d in n]
    H = int(np.prod([c + 2 for c in nc]))
    assert starts.size == stops.size == H
    # the reference's own assertion (test_particles.jl:85)
    assert int(np.sum(stops - starts + 1)) == npart
    assert np.all(np.diff(hashes) >= 0)
    pos = (_abi.PROP_X, _abi.PROP_Y, _abi.PROP_Z) if stage == 1 else (_abi.PROP_X2, _abi.PROP_Y2, _abi.PROP_Z2)
    h0 = cell_hash(*(before[p] for p in pos), n, ratio)
    perm = np.argsort(h0, kind="stable")
    assert np.array_equal(hashes, h0[perm])
    ids = e.download_particles(0)["ids"]
    assert np.array_equal(ids, perm + 1)  # ids were 1..n: a stable sort keeps ties ascending
    for p in range(_abi.NPROP):
        assert np.array_equal(e.prop_get(0, p), before[p][perm]), p
    xs = np.arange(1, H + 1)
    assert np.array_equal(starts, np.searchsorted(hashes, xs, side="left") + 1)
    assert np.array_equal(stops, np.searchsorted(hashes, xs, side="right"))
    return hashes, starts, stops


def test_reference_setup_invariant():
    """test_particles.jl:79-91: 16^3 grid, Cell(4), 10 particles."""
    n = (16, 16, 16)
    e, before = setup(n, 10, 0, 4)
    check_index(e, before, n, 4, 1)
    e.close()


@pytest.mark.parametrize("n,ratio,npart,stage", [((16, 16, 16), 1, 500, 1), ((24, 16, 20), 2, 2000, 2),
                                                 ((32, 32, 32), 4, 5000, 1), ((16, 16, 16), 8, 300, 2)])
def test_index_properties(n, ratio, npart, stage):
    e, before = setup(n, npart, 1 + ratio, ratio)
    check_index(e, before, n, ratio, stage)
    e.close()


def test_positions_on_cell_faces_and_many_ties():
    """Positions exactly on cell boundaries (k * dxc, 0) and many particles per
    cell: the floor of an exact multiple and the order of ties."""
    n, ratio, npart = (16, 16, 16), 4, 400
    rng = np.random.default_rng(7)
    dxc = (L / 16) * ratio
    x = rng.integers(0, 4, npart) * dxc
    y = np.where(rng.random(npart) < 0.5, 0.0, rng.integers(0, 4, npart) * dxc)
    z = rng.integers(0, 2, npart) * dxc + 1e-3
    e, before = setup(n, npart, 7, ratio, positions=[x, y, z])
    hashes, starts, stops = check_index(e, before, n, ratio, 1)
    assert np.unique(hashes).size <= 4 * 4 * 2  # ties in every occupied cell
    e.close()


def out_of_domain_positions(npart, seed):
    """Positions a step can leave before the next boundary! pass: just below 0,
    on 0 and 2pi, just below and above 2pi (halo cells 0 and nc+1 of each axis)."""
    rng = np.random.default_rng(seed)
    edge = np.array([-1e-12, -0.05, 0.0, np.nextafter(L, 0.0), L, L + 1e-12, L + 0.05, np.nextafter(0.0, -1.0)])
    out = []
    for _ in range(3):
        a = rng.random(npart) * L
        pick = rng.random(npart) < 0.6
        a[pick] = rng.choice(edge, int(pick.sum()))
        out.append(a)
    return out


def test_positions_outside_the_domain():
    """Hashes in the halo cells 0 and nc+1 (hash axes 0:nc+1, hasher.jl:15-38)."""
    n, ratio, npart = (16, 16, 16), 4, 600
    e, before = setup(n, npart, 9, ratio, positions=out_of_domain_positions(npart, 9))
    hashes, _, _ = check_index(e, before, n, ratio, 1)
    nc = 16 // ratio
    assert hashes.min() == 1 and hashes.max() == (nc + 2) ** 3  # both corner halo cells are used
    e.close()


def test_index_errors():
    e, _ = setup((16, 16, 16), 10, 0, 4)
    with pytest.raises(Exception) as exc:
        e.particles_cellindex(0, 4)
    assert getattr(exc.value, "code", None) == _abi.ESTATE
    for bad in (0, 3, 32):
        with pytest.raises(Exception) as exc:
            e.particles_makeindex(0, 1, bad)
        assert getattr(exc.value, "code", None) == _abi.EINVAL
    with pytest.raises(Exception):
        e.particles_makeindex(0, 3, 4)
    e.close()
