"""Shared cases of the batching and serving tests: they run over the CPU oracle
(tests/test_serve.py, no GPU) and over the CUDA library (tests/test_gpu_serve.py).

Every case compares a run driven by the batch or the server with the same run
alone on its own handle, from identical inputs.  The kernels are deterministic
and a member's arithmetic does not depend on the others, so the comparison is
exact (==) in both precision forms.
"""

import numpy as np

from helpers import make_config
from lcs_b200 import Batch, Server, _abi, inits

F = _abi


def same_log(a, b):
    """Step logs equal field by field (NaN == NaN: runs without forcing log NaN power)."""
    def flat(d, pre=""):
        out = {}
        for k, v in d.items():
            if isinstance(v, dict):
                out.update(flat(v, pre + k + "."))
            else:
                out[pre + k] = v
        return out
    fa, fb = flat(a), flat(b)
    return fa.keys() == fb.keys() and all(
        (fa[k] == fb[k]) or (isinstance(fa[k], float) and np.isnan(fa[k]) and np.isnan(fb[k])) for k in fa)


def same_logs(a, b):
    return len(a) == len(b) and all(same_log(x, y) for x, y in zip(a, b))


def member_configs(precision=F.PRECISION_FP64):
    """Uneven sizes, particle counts and parameters (the batching form's shape)."""
    return [
        make_config(16, species=[{"n": 300, "density_ratio": 843.0}], Re=80.0, itrmax=8, precision=precision),
        make_config(dims=(24, 16, 20), mode=F.MODE_FLOW, Re=40.0, itrmax=7, precision=precision),
        make_config(16, species=[{"n": 120, "density_ratio": 100.0}, {"n": 200, "density_ratio": 843.0}],
                    forcing=F.FORCING_LINEAR_POWER, power=0.5, Re=60.0, itrmax=9, precision=precision),
    ]


def group_configs(precision=F.PRECISION_FP64, n=24, count=4):
    """Members of one shape (the grouped form): different viscosity, forcing,
    particle counts and species; same dims, halo and HSMAC settings."""
    kinds = [
        dict(species=[{"n": 300, "density_ratio": 843.0}], Re=80.0),
        dict(species=[{"n": 120, "density_ratio": 100.0}, {"n": 200, "density_ratio": 843.0}],
             forcing=F.FORCING_LINEAR_POWER, power=0.5, Re=60.0),
        dict(mode=F.MODE_FLOW, Re=40.0),
        dict(species=[{"n": 500, "density_ratio": 843.0}], forcing=F.FORCING_LINEAR_POWER, power=0.3, Re=120.0),
    ]
    return [make_config(n, itrmax=8, precision=precision, **kinds[i % len(kinds)]) for i in range(count)]


def load_inputs(e, cfg, seed):
    flow, parts = inputs(cfg, seed)
    e.upload_flow(*flow)
    for s, p in enumerate(parts):
        e.upload_particles(s, p["diam"], p["x"], p["y"], p["z"], p["u"], p["v"], p["w"])
        e.init_particle_velocity(s)


def check_group_equals_members_alone(engine_cls, lib, precision=F.PRECISION_FP64, count=4, nsteps=3, n=24):
    """lcs_group_create over handles of one shape: each member's fields,
    particles and logs equal the member stepped alone, bit for bit."""
    import ctypes as C

    cfgs = group_configs(precision, n=n, count=count)
    engines = [engine_cls(c) for c in cfgs]
    for i, (c, e) in enumerate(zip(cfgs, engines)):
        load_inputs(e, c, 200 + i)
    hs = (C.c_void_p * count)(*[e.handle.value for e in engines])
    grp = C.c_void_p()
    assert lib.lcs_group_create(hs, count, C.byref(grp)) == 0, lib.lcs_last_error(None)
    logs = []
    for rep in range(2):  # the second round replays the captured group graph
        assert lib.lcs_group_step_begin(grp, nsteps) == 0, lib.lcs_last_error(None)
        for e in engines:
            lg = (_abi.Log * nsteps)()
            e._check(lib.lcs_step_finish(e.handle, lg))
            if rep == 1:
                logs.append([x.as_dict() for x in lg])
    lib.lcs_group_destroy(grp)
    for i, (c, e) in enumerate(zip(cfgs, engines)):
        c.use_graphs = 1
        flow, parts, ref_logs = run_alone(engine_cls, c, 200 + i, 2 * nsteps)
        assert same_logs(logs[i], ref_logs[nsteps:]), i
        for a, r in zip(e.download_flow(), flow):
            assert np.array_equal(a, r), i
        for s in range(len(parts)):
            got = e.download_particles(s)
            for k in ("x", "y", "z", "u", "v", "w"):
                assert np.array_equal(got[k], parts[s][k]), (i, s, k)
        e.close()


def inputs(cfg, seed):
    """Seeded initial state of one run: interior fields and particle species."""
    nx, ny, nz = (int(d) for d in cfg.dims)
    rng = np.random.default_rng(seed)
    flow = [rng.standard_normal((nz, ny, nx)) * 0.3 for _ in range(4)]
    flow[3] *= 0.0
    parts = []
    if cfg.mode == F.MODE_FLOW_PARTICLE:
        for s in range(int(cfg.n_species)):
            n = int(cfg.species[s].nvalid)
            x, y, z = inits.random_positions(n, seed * 10 + s)
            zero = np.zeros(n)
            parts.append({"diam": np.full(n, 0.01 * (s + 1)), "x": x, "y": y, "z": z, "u": zero, "v": zero, "w": zero})
    return flow, parts


def run_alone(engine_cls, cfg, seed, nsteps, tuning=None):
    e = engine_cls(cfg)
    if tuning is not None:  # the launch shapes the batch gave this member
        e._check(e.lib.lcs_set_tuning(e.handle, tuning["rw_rows"], tuning["zchunk"], tuning["share"]))
    flow, parts = inputs(cfg, seed)
    e.upload_flow(*flow)
    for s, p in enumerate(parts):
        e.upload_particles(s, p["diam"], p["x"], p["y"], p["z"], p["u"], p["v"], p["w"])
        e.init_particle_velocity(s)
    logs = e.step(nsteps)
    out = (e.download_flow(), [e.download_particles(s) for s in range(len(parts))], logs)
    e.close()
    return out


def check_async_equals_step(engine_cls, lib):
    cfg = member_configs()[0]
    cfg.use_graphs = 1
    ref = run_alone(engine_cls, cfg, 3, 3)
    e = engine_cls(cfg)
    flow, parts = inputs(cfg, 3)
    e.upload_flow(*flow)
    for s, p in enumerate(parts):
        e.upload_particles(s, p["diam"], p["x"], p["y"], p["z"], p["u"], p["v"], p["w"])
        e.init_particle_velocity(s)
    e._check(lib.lcs_step_begin(e.handle, 2))
    import ctypes as C

    done = C.c_int32()
    e._check(lib.lcs_step_poll(e.handle, C.byref(done)))
    assert lib.lcs_step_begin(e.handle, 1) == F.ESTATE  # one batch of steps in flight at a time
    logs = (_abi.Log * 2)()
    e._check(lib.lcs_step_finish(e.handle, logs))
    e._check(lib.lcs_step_begin(e.handle, 1))
    logs1 = (_abi.Log * 1)()
    e._check(lib.lcs_step_finish(e.handle, logs1))
    got = [logs[0].as_dict(), logs[1].as_dict(), logs1[0].as_dict()]
    assert [g["step"] for g in got] == [1, 2, 3]
    assert same_logs(got, ref[2])
    for a, b in zip(e.download_flow(), ref[0]):
        assert np.array_equal(a, b)
    e.close()


def check_batch_equals_members_alone(engine_cls, lib, precision=F.PRECISION_FP64, nsteps=3, cfgs=None):
    cfgs = member_configs(precision) if cfgs is None else cfgs
    b = Batch(cfgs, lib=lib)
    for i, (cfg, e) in enumerate(zip(cfgs, b.members)):
        flow, parts = inputs(cfg, 100 + i)
        e.upload_flow(*flow)
        for s, p in enumerate(parts):
            e.upload_particles(s, p["diam"], p["x"], p["y"], p["z"], p["u"], p["v"], p["w"])
            e.init_particle_velocity(s)
    logs = b.step(nsteps)
    for i, (cfg, e) in enumerate(zip(cfgs, b.members)):
        cfg_alone = cfgs[i]
        cfg_alone.use_graphs = 1
        # launch shapes change only the grouping of the residual's partial sums:
        # the solo run uses the member's shapes, and then every bit agrees
        flow, parts, ref_logs = run_alone(engine_cls, cfg_alone, 100 + i, nsteps, tuning=b.tuning(i))
        assert same_logs(logs[i], ref_logs)
        for a, r in zip(e.download_flow(), flow):
            assert np.array_equal(a, r)
        for s in range(len(parts)):
            got = e.download_particles(s)
            for k in ("x", "y", "z", "u", "v", "w"):
                assert np.array_equal(got[k], parts[s][k])
    b.close()


def check_server(engine_cls, lib, precision=F.PRECISION_FP64, device=0):
    """Five requests, two slots, a budget that holds about two runs: requests
    queue, are admitted as runs finish, and each result equals its solo run.
    A request larger than the whole budget fails with ENOMEM."""
    cfgs = member_configs(precision)
    jobs = [(cfgs[0], 1, 4), (cfgs[1], 2, 2), (cfgs[2], 3, 3), (cfgs[0], 4, 1), (cfgs[1], 5, 0)]
    fp = [engine_footprint(lib, c) for c, _, _ in jobs]
    budget = sorted(fp)[-1] + sorted(fp)[-2]
    srv = Server(device=device, max_active=2, steps_per_slice=2, hbm_budget_bytes=budget, lib=lib)
    tickets = []
    for cfg, seed, n in jobs:
        flow, parts = inputs(cfg, seed)
        tickets.append(srv.submit(cfg, *flow, species=parts, nsteps=n, interp_velocity=True))
    big = make_config(64, mode=F.MODE_FLOW, precision=precision)
    flow_big = [np.zeros((64, 64, 64)) for _ in range(4)]
    t_big = srv.submit(big, *flow_big, nsteps=1)
    srv.drain(600.0)
    st = srv.stats()
    assert st["completed"] == len(jobs) and st["failed"] == 1 and st["queued"] == 0 and st["active"] == 0
    assert 0 < st["peak_bytes_in_use"] <= budget
    assert 0 < st["p50_latency_s"] <= st["p99_latency_s"]
    state, _ = srv.poll(t_big)
    assert state == F.REQ_FAILED
    try:
        srv.result(t_big)
        raise AssertionError("the over-budget request returned a result")
    except Exception as exc:  # LCSError(ENOMEM)
        assert getattr(exc, "code", None) == F.ENOMEM
    for t, (cfg, seed, n) in zip(tickets, jobs):
        state, done = srv.poll(t)
        assert state == F.REQ_DONE and done == n
        res = srv.result(t)
        c = cfg
        c.use_graphs = 1
        flow, parts, logs = run_alone(engine_cls, c, seed, n)
        for a, r in zip(res["flow"], flow):
            assert np.array_equal(a, r)
        for s in range(len(parts)):
            for k in ("x", "y", "z", "u", "v", "w"):
                assert np.array_equal(res["particles"][s][k], parts[s][k])
        if n:
            assert same_log(res["log"], logs[-1])
        assert res["latency_s"] > 0
        srv.release(t)
    srv.close()


def engine_footprint(lib, cfg):
    import ctypes as C

    b = C.c_int64()
    assert lib.lcs_footprint(C.byref(cfg), C.byref(b)) == 0
    return b.value
