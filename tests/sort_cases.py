"""Cases of the particle sort (lcs_set_particle_sort), shared by the oracle and
GPU tests.

The sort runs makeindex! (src/particles/makeindex.jl:29-67) on every species
after every interval-th step.  Each particle's arithmetic (boundary!, motion!,
update!: src/particles/{boundary,motion,update}.jl) reads only its own values
and the fluid, so sorting changes the order of the arrays and nothing else: a
particle, matched by its id, has the same bits as in the unsorted run, and the
flow is untouched.
"""

import ctypes as C
import math

import numpy as np

from helpers import make_config
from lcs_b200 import _abi
from serve_cases import inputs

L = 2 * math.pi


def sort_config(n=16, graphs=0, precision=_abi.PRECISION_FP64):
    """Two species, no forcing and a fixed 8 sweeps per couple (epsp below any
    residual), so that the CUDA library and the oracle agree bit for bit."""
    return make_config(n, species=[{"n": 700, "density_ratio": 843.0}, {"n": 400, "density_ratio": 100.0}],
                       itrmax=8, epsp=1e-30, Re=50.0, graphs=graphs, precision=precision)


def cell_hashes(x, y, z, dims, ratio):
    """The makeindex! hash (makeindex.jl:45-52, hasher.jl:15-38): 1-based
    column-major index of floor(x / dxc) + 1 over the cell axes 0:nc+1."""
    h = np.ones(x.shape, np.int64)
    stride = 1
    for a, c in enumerate((x, y, z)):
        nc = dims[a] // ratio
        dxc = (L / dims[a]) * ratio
        h += (np.floor(c / dxc).astype(np.int64) + 1) * stride
        stride *= nc + 2
    return h


def run(engine_cls, cfg, seed, nsteps, interval, ratio=4, use_async=False):
    """nsteps steps of one run (lcs_step, or lcs_step_begin/finish), with the
    particle sort every `interval` steps (0: none); the final state."""
    e = engine_cls(cfg)
    flow, parts = inputs(cfg, seed)
    e.upload_flow(*flow)
    for s, p in enumerate(parts):  # ids 1..n, so that particles can be matched after a sort
        n = p["x"].size
        e.upload_particles(s, p["diam"], p["x"], p["y"], p["z"], p["u"], p["v"], p["w"], ids=np.arange(1, n + 1))
        e.init_particle_velocity(s)
    if interval:
        e.set_particle_sort(interval, ratio)
    if use_async:
        e._check(e.lib.lcs_step_begin(e.handle, nsteps))
        e._check(e.lib.lcs_step_finish(e.handle, None))
    else:
        e.step(nsteps)
    out = {"flow": e.download_flow(), "parts": [e.download_particles(s) for s in range(int(cfg.n_species))]}
    e.close()
    return out


def by_id(p):
    o = np.argsort(p["ids"], kind="stable")
    return {k: v[o] for k, v in p.items()}


def check_sort_keeps_values(engine_cls, nsteps=4, interval=2, ratio=4, graphs=0, use_async=False,
                            precision=_abi.PRECISION_FP64):
    """The sorted run equals the unsorted one particle by particle (by id) and
    field by field, bit for bit; after a sort step the order is by cell."""
    cfg = sort_config(graphs=graphs, precision=precision)
    a = run(engine_cls, cfg, 7, nsteps, 0, use_async=use_async)
    b = run(engine_cls, cfg, 7, nsteps, interval, ratio, use_async=use_async)
    for fa, fb in zip(a["flow"], b["flow"]):
        assert np.array_equal(fa, fb)
    dims = [int(d) for d in cfg.dims]
    for s, (pa, pb) in enumerate(zip(a["parts"], b["parts"])):
        qa, qb = by_id(pa), by_id(pb)
        for k in qa:
            assert np.array_equal(qa[k], qb[k]), (s, k)
        assert not np.array_equal(pa["ids"], pb["ids"]), "the sort left the upload order"
        if nsteps % interval == 0:  # the last step was followed by a sort
            h = cell_hashes(pb["x"], pb["y"], pb["z"], dims, ratio)
            assert np.all(np.diff(h) >= 0), s
    return b


def check_group_sort_equals_alone(engine_cls, lib, nsteps=3):
    """A batch group (lcs_group_create) whose second member sorts every step:
    each member's fields and particles (in their order) equal the member
    stepped alone with the same sort setting, bit for bit."""
    cfg = sort_config()
    setting = [0, 1]

    def start(i):
        e = engine_cls(cfg)
        flow, parts = inputs(cfg, 40 + i)
        e.upload_flow(*flow)
        for s, p in enumerate(parts):
            n = p["x"].size
            e.upload_particles(s, p["diam"], p["x"], p["y"], p["z"], p["u"], p["v"], p["w"], ids=np.arange(1, n + 1))
            e.init_particle_velocity(s)
        if setting[i]:
            e.set_particle_sort(setting[i], 4)
        return e

    def state(e):
        return e.download_flow(), [e.download_particles(s) for s in range(int(cfg.n_species))]

    alone = []
    for i in range(2):
        e = start(i)
        e._check(e.lib.lcs_step_begin(e.handle, nsteps))
        e._check(e.lib.lcs_step_finish(e.handle, None))
        alone.append(state(e))
        e.close()
    engines = [start(i) for i in range(2)]
    hs = (C.c_void_p * 2)(*[e.handle.value for e in engines])
    grp = C.c_void_p()
    assert lib.lcs_group_create(hs, 2, C.byref(grp)) == 0, lib.lcs_last_error(None)
    try:
        assert lib.lcs_group_step_begin(grp, nsteps) == 0, lib.lcs_last_error(None)
        for e in engines:
            e._check(lib.lcs_step_finish(e.handle, None))
        for i, e in enumerate(engines):
            flow, parts = state(e)
            for a, b in zip(flow, alone[i][0]):
                assert np.array_equal(a, b), i
            for s, (pa, pb) in enumerate(zip(parts, alone[i][1])):
                for k in pa:
                    assert np.array_equal(pa[k], pb[k]), (i, s, k)
        assert not np.array_equal(alone[1][1][0]["ids"], np.arange(1, alone[1][1][0]["ids"].size + 1))
    finally:
        lib.lcs_group_destroy(grp)
        for e in engines:
            e.close()
