"""The `.lcs-yaml` reader (LCSIO.readconfig, src/LCSIO/config.jl:6-31, with the
kind-tagged objects of lib/polyserde/src/PolySerde.jl:35-80) and the
`LCS.simulate` mirror (src/simulate.jl:13-90), over the CPU oracle."""

import math
import os

import numpy as np
import pytest
import yaml

from lcs_b200 import _abi, config as lcfg
from lcs_b200.simulate import init_engine, simulate
from oracle_engine import OracleEngine


def reference_style(n=16):
    """A config in the reference's schema (field names of src/config.jl,
    src/flows/config.jl, src/particles/config.jl), with settings that differ
    from the workload builder's defaults."""
    return {
        "outdir": "output",
        "mode": {"kind": "flow-particle"},
        "backend": {"kind": "cuda"},
        "topo": {"proc_dims": [0, 0, 0], "reorder": False},
        "grid": {"dims": [n, n, n], "halo_size": 3},
        "timestep": {"cfl": 0.25, "dtmax": 0.005},
        "simulate": {"last_step": 4, "interval_stat": 3, "interval_restart": 100},
        "flow": {
            "params": {"U0_m_s": 2.0, "L0_m": 0.5, "NU_m2_s": 0.01},
            "init": {"kind": "spectral", "params": {"seed": 4, "urms": 1.0, "kpeak": 3.0}},
            "couple": {"kind": "hsmac", "params": {
                "time_blocking": False, "overlap": True, "coloring": {"kind": "red-black-block", "params": {"size": 2}},
                "omega": 1.5, "epsp": 1e-6, "itrmin": 4, "itrmax": 9}},
            "forcing": {"kind": "rc-energy", "params": {"kmin": 1, "kmax": 2, "energy": 0.649, "coarse_size": 4}},
        },
        "particles": [
            {"population": {"valid": 50, "invalid_ratio": 0.0},
             "params": {"gravity": 0.0, "density_ratio": 843.0}, "drag": {"kind": "nonlinear"},
             "init": {"position": {"kind": "random", "params": {"seed": 3}}, "velocity": {"kind": "interp"},
                      "size": {"kind": "const", "params": {"diam_m": 0.01}}}},
            {"population": {"valid": 30}, "params": {"gravity": 9.8, "density_ratio": 100.0},
             "init": {"size": {"kind": "const", "params": {"diam_m": 0.002}}}},
        ],
    }


def test_readconfig_maps_every_field(tmp_path):
    p = tmp_path / "run.lcs-yaml"
    p.write_text(yaml.safe_dump(reference_style()))
    rc = lcfg.readconfig(str(p))
    c = rc.abi
    assert rc.dims == (16, 16, 16) and c.halo_size == 3
    assert (c.cfl, c.dtmax) == (0.25, 0.005)
    assert (c.U0, c.L0, c.NU) == (2.0, 0.5, 0.01)
    assert c.mode == _abi.MODE_FLOW_PARTICLE and c.precision == _abi.PRECISION_FP64
    assert (c.time_blocking, c.overlap) == (0, 1)
    assert c.coloring == _abi.COLORING_RED_BLACK_BLOCK and c.coloring_block == 2
    assert (c.omega, c.epsp, c.itrmin, c.itrmax) == (1.5, 1e-6, 4, 9)
    assert c.forcing == _abi.FORCING_RC_ENERGY
    assert (c.kmin, c.kmax, c.coarse_size, c.energy) == (1, 2, 4, 0.649)
    assert c.n_species == 2
    assert (c.species[0].nvalid, c.species[0].drag, c.species[0].density_ratio) == (50, _abi.DRAG_NONLINEAR, 843.0)
    assert (c.species[1].nvalid, c.species[1].drag, c.species[1].gravity) == (30, _abi.DRAG_LINEAR, 9.8)
    # the non-dimensional diameter diam_m / L0 (particles/config.jl:233)
    assert rc.species[0].diam == 0.01 / 0.5 and rc.species[1].diam == 0.002 / 0.5
    assert rc.species[0].velocity == "interp" and rc.species[1].velocity == "rest"
    assert rc.species[0].position_seed == 3
    assert (rc.last_step, rc.interval_stat) == (4, 3)
    assert rc.flow_init == "spectral" and rc.flow_init_params["kpeak"] == 3.0


def test_workload_builder_round_trips_through_yaml(tmp_path):
    d = lcfg.workload(32, 0.005, {"kind": "linear-power", "params": {"power": 0.5}}, [0.05, 0.5], [100, 200],
                      precision="fp32-mixed", itrmax=50, steps=7)
    p = tmp_path / "w.lcs-yaml"
    p.write_text(yaml.safe_dump(d))
    rc = lcfg.readconfig(str(p))
    c = rc.abi
    assert c.precision == _abi.PRECISION_FP32_MIXED and c.forcing == _abi.FORCING_LINEAR_POWER and c.power == 0.5
    assert c.NU == 0.005 and c.itrmax == 50 and rc.last_step == 7
    assert math.isclose(c.epsp, 1e-8 * 2 * math.pi / 32)
    Re = 1.0 / 0.005
    for s, tp in enumerate((0.05, 0.5)):
        assert math.isclose(lcfg.taup(843.0, Re, rc.species[s].diam), tp, rel_tol=1e-12)


@pytest.mark.parametrize("edit,msg", [
    (lambda d: d["flow"]["couple"].__setitem__("kind", "sor"), "couple kind"),
    (lambda d: d["grid"].__setitem__("dims", [16, 16]), "3 entries"),
    (lambda d: d["particles"][0]["init"].__setitem__("size", {"kind": "uniform"}), "size init"),
    (lambda d: d.__setitem__("backend", {"kind": "tpu"}), "backend kind"),
    (lambda d: d.__setitem__("particles", d["particles"] * 9), "species"),
])
def test_config_errors(edit, msg):
    d = reference_style()
    edit(d)
    with pytest.raises(ValueError) as exc:
        lcfg.from_dict(d)
    assert msg in str(exc.value)


def small_run(n=16, steps=3, interval=2):
    d = lcfg.workload(n, 0.01, {"kind": "linear-power", "params": {"power": 0.5}}, [0.1, 0.5], [200, 100],
                      itrmax=12, steps=steps)
    d["simulate"]["interval_stat"] = interval
    return d


def test_simulate_equals_a_manual_step_loop():
    """simulate() = init + `lcs_step` in interval_stat chunks: the same logs and
    final state as one loop of timestep! + evolve! over the same init."""
    d = small_run()
    eng, logs = simulate(d, quiet=True, engine_cls=OracleEngine)
    # `for _ in state.step:last_step` (src/simulate.jl:54) from step 0: last_step + 1 steps
    assert [lg["step"] for lg in logs] == [1, 2, 3, 4]
    ref = init_engine(lcfg.from_dict(d), OracleEngine)
    manual = []
    for _ in range(4):
        dt = ref.timestep()
        manual.append((dt, ref.evolve(dt)))
    for lg, (dt, ev) in zip(logs, manual):
        assert lg["dt"] == dt
        assert lg["couple1"]["itr"] == ev["couple1"]["itr"] and lg["couple2"]["div"] == ev["couple2"]["div"]
    for a, b in zip(eng.download_flow(), ref.download_flow()):
        assert np.array_equal(a, b)
    for s in range(2):
        pa, pb = eng.download_particles(s), ref.download_particles(s)
        for k in pa:
            assert np.array_equal(pa[k], pb[k]), (s, k)
    # generated ids run on across species (particles/init.jl)
    ids = np.concatenate([eng.download_particles(s)["ids"] for s in range(2)])
    assert np.array_equal(np.sort(ids), np.arange(1, 301))
    eng.close()
    ref.close()


def test_simulate_prints_one_line_per_step(capsys):
    eng, logs = simulate(small_run(steps=2, interval=5), engine_cls=OracleEngine)
    out = capsys.readouterr().out.strip().splitlines()
    assert len(out) == 3 and out[0].startswith("step=1 ") and "couple1=(itr=" in out[0]
    eng.close()


def test_simulate_writes_stat_and_restart_files(tmp_path):
    """save=True: stat.h5 gets one entry per interval_stat step (the savestat
    tree), restart.h5.<step> every interval_restart steps with the oldest
    beyond num_restart_files removed (LCSIO.cleanrestart), and the last restart
    reloads to the run's final state."""
    from lcs_b200 import restart
    from oracle_engine import load_oracle

    d = small_run(steps=5, interval=2)  # steps 1..6
    d["simulate"].update({"interval_restart": 3, "num_restart_files": 1})
    for p in d["particles"]:
        p["cell"] = {"grid_ratio": 2}
        p["stat"] = {"rdf": {"contact_tolerance": 0.01, "bin_size": 4, "min_radius": 1e-3, "search_cell_size": 1},
                     "spectrum": {"max_wavenumber": 6, "nsamples": 8}}
    rc = lcfg.from_dict(d)
    assert rc.species[0].grid_ratio == 2 and rc.species[1].spectrum["nsamples"] == 8
    eng, logs = simulate(rc, quiet=True, engine_cls=OracleEngine, save=True, outdir=str(tmp_path))
    lib = load_oracle()
    files = sorted(os.listdir(tmp_path))
    assert files == ["restart.h5.6", "stat.h5"]
    stat = str(tmp_path / "stat.h5")
    assert restart.listing(lib, stat) == ["2", "4", "6"]
    assert restart.dataset(lib, stat, "4/stat/state/step").tolist() == 4
    assert restart.dataset(lib, stat, "6/log/flow/couple1/itr").tolist() == logs[5]["couple1"]["itr"]
    assert restart.dataset(lib, stat, "6/log/flow/forcing/p").tolist() == logs[5]["forcing"]["p"]
    assert restart.dataset(lib, stat, "6/state/particles/2/nvalid").tolist() == 100
    k = restart.dataset(lib, stat, "2/stat/particles/1/spectrum/wavenumbers")
    assert k.size == restart.dataset(lib, stat, "2/stat/particles/1/spectrum/Enp").size and k.max() == 6
    fresh = OracleEngine(rc.abi)
    restart.load(fresh, str(tmp_path / "restart.h5.6"))
    for a, b in zip(fresh.download_flow(), eng.download_flow()):
        assert np.array_equal(a, b)
    for s in range(2):
        pa, pb = fresh.download_particles(s), eng.download_particles(s)
        for k in pa:
            assert np.array_equal(pa[k], pb[k]), (s, k)
    fresh.close()
    eng.close()


def test_resume_continues_the_run(tmp_path):
    """LCS_RESUME: a run stopped at step 4 (last_step 3; restart.h5.3, stat.h5)
    and resumed from step 3 to step 7 (last_step 6) ends where an uninterrupted
    run ends (flow bit for bit,
    particles by id), with the step counter and time carried over."""
    d = small_run(steps=3, interval=3)
    d["simulate"].update({"interval_restart": 3, "num_restart_files": 2})
    out = str(tmp_path / "run")
    eng, _ = simulate(d, quiet=True, engine_cls=OracleEngine, save=True, outdir=out)
    eng.close()
    d6 = small_run(steps=6, interval=3)
    d6["simulate"].update({"interval_restart": 3, "num_restart_files": 2})
    resumed, rlogs = simulate(d6, quiet=True, engine_cls=OracleEngine, save=True, outdir=out, resume=True)
    assert [lg["step"] for lg in rlogs] == [4, 5, 6, 7]
    assert sorted(os.listdir(out)) == ["restart.h5.3", "restart.h5.6", "stat.h5"]
    whole, wlogs = simulate(d6, quiet=True, engine_cls=OracleEngine)
    assert rlogs[-1]["t"] == wlogs[-1]["t"] and resumed.get_state() == whole.get_state()
    for a, b in zip(resumed.download_flow(), whole.download_flow()):
        assert np.array_equal(a, b)
    for s in range(2):
        pa, pb = resumed.download_particles(s), whole.download_particles(s)
        oa, ob = np.argsort(pa["ids"]), np.argsort(pb["ids"])
        for k in pa:
            assert np.array_equal(pa[k][oa], pb[k][ob]), (s, k)
    with pytest.raises(ValueError):
        simulate(d6, quiet=True, engine_cls=OracleEngine, outdir=str(tmp_path / "empty"), resume=True)
    resumed.close()
    whole.close()


def test_restart_and_upsample_inits(tmp_path):
    """flow.init restart / upsample and the particles' restart kinds
    (ParticleRestart(file, iprofile)) read a restart file through the library."""
    from lcs_b200 import restart

    d = small_run(steps=2, interval=2)
    eng, _ = simulate(d, quiet=True, engine_cls=OracleEngine)
    f = str(tmp_path / "restart.h5.2")
    restart.save(eng, f)
    r = small_run()
    r["flow"]["init"] = {"kind": "restart", "params": {"file": f}}
    for i, p in enumerate(r["particles"]):
        rk = {"kind": "restart", "params": {"file": f, "iprofile": i + 1}}
        p["init"] = {"id": rk, "position": rk, "velocity": rk, "size": rk}
    again = init_engine(lcfg.from_dict(r), OracleEngine)
    for a, b in zip(again.download_flow(), eng.download_flow()):
        assert np.array_equal(a, b)
    for s in range(2):
        pa, pb = again.download_particles(s), eng.download_particles(s)
        for k in pa:
            assert np.array_equal(pa[k], pb[k]), (s, k)
    up = small_run(n=32)
    up["flow"]["init"] = {"kind": "upsample", "params": {"file": f}}
    fine = init_engine(lcfg.from_dict(up), OracleEngine)
    ref = OracleEngine(lcfg.from_dict(small_run(n=32)).abi)
    restart.load_coarse(ref, f)
    for a, b in zip(fine.download_flow(), ref.download_flow()):
        assert np.array_equal(a, b)
    for e in (eng, again, fine, ref):
        e.close()


def test_command_line_run_and_resume(tmp_path, monkeypatch, capsys):
    """python -m lcs_b200 cfg [steps]: a fresh output directory with the
    config saved, refusal of an existing one without LCS_RESUME, and a resume."""
    from lcs_b200 import restart
    from lcs_b200.simulate import main
    from oracle_engine import load_oracle

    d = small_run(steps=4, interval=2)
    d["simulate"].update({"interval_restart": 2, "num_restart_files": 1})
    out = tmp_path / "out"
    d["outdir"] = str(out)
    cfg = tmp_path / "run.lcs-yaml"
    cfg.write_text(yaml.safe_dump(d))
    monkeypatch.delenv("LCS_RESUME", raising=False)
    assert main([str(cfg), "2"], engine_cls=OracleEngine) == 0
    assert sorted(os.listdir(out)) == ["config.lcs-yaml", "restart.h5.2", "stat.h5"]
    assert yaml.safe_load((out / "config.lcs-yaml").read_text())["simulate"]["last_step"] == 4
    with pytest.raises(ValueError, match="LCS_RESUME"):
        main([str(cfg)], engine_cls=OracleEngine)
    monkeypatch.setenv("LCS_RESUME", "1")
    assert main([str(cfg)], engine_cls=OracleEngine) == 0  # steps 3, 4 and 5 (state.step 2 : last_step 4)
    assert sorted(os.listdir(out)) == ["config.lcs-yaml", "restart.h5.4", "stat.h5"]
    assert restart.listing(load_oracle(), str(out / "stat.h5")) == ["2", "4"]
    lines = [x for x in capsys.readouterr().out.splitlines() if x.startswith("step=")]
    assert [x.split()[0] for x in lines] == ["step=1", "step=2", "step=3", "step=4", "step=5"]


def test_backend_particle_sort_param():
    """backend.params.particle_sort: the run sorts its particles by cell and
    each particle (by id) and the flow equal the unsorted run's."""
    d = small_run(steps=2, interval=5)
    plain, _ = simulate(d, quiet=True, engine_cls=OracleEngine)
    d["backend"]["params"]["particle_sort"] = 1
    for p in d["particles"]:
        p["cell"] = {"grid_ratio": 4}
    rc = lcfg.from_dict(d)
    assert rc.particle_sort == 1
    sorted_, _ = simulate(rc, quiet=True, engine_cls=OracleEngine)
    for a, b in zip(plain.download_flow(), sorted_.download_flow()):
        assert np.array_equal(a, b)
    for s in range(2):
        pa, pb = plain.download_particles(s), sorted_.download_particles(s)
        assert not np.array_equal(pa["ids"], pb["ids"])
        oa, ob = np.argsort(pa["ids"]), np.argsort(pb["ids"])
        for k in pa:
            assert np.array_equal(pa[k][oa], pb[k][ob]), (s, k)
    plain.close()
    sorted_.close()
