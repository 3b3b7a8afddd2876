"""Restart files between the CUDA library and the oracle: a state saved by one
loads into the other bit for bit, in both precision forms (the FP32-mixed
form saves its FP32 fields as the Float64 values they are)."""

import math

import numpy as np
import pytest

from helpers import make_config
from lcs_b200 import Engine, _abi, restart
from oracle_engine import OracleEngine

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_FP32_MIXED])
def test_gpu_restart_loads_into_oracle_and_back(tmp_path, precision):
    cfg = make_config(32, species=[{"n": 2000, "density_ratio": 843.0}, {"n": 500, "density_ratio": 100.0}],
                      Re=80.0, itrmax=8, precision=precision)
    g = Engine(cfg)
    rng = np.random.default_rng(7)
    g.upload_flow(*[rng.standard_normal((32, 32, 32)) * 0.3 for _ in range(3)], np.zeros((32, 32, 32)))
    for s, m in enumerate((2000, 500)):
        pos = [rng.random(m) * 2 * math.pi for _ in range(3)]
        g.upload_particles(s, np.full(m, 0.01), *pos, *[np.zeros(m)] * 3, ids=np.arange(1, m + 1))
        g.init_particle_velocity(s)
    g.step(3)
    path = str(tmp_path / "restart.h5.3")
    restart.save(g, path)
    ocfg = make_config(32, species=[{"n": 2000, "density_ratio": 843.0}, {"n": 500, "density_ratio": 100.0}],
                       Re=80.0, itrmax=8)
    o = OracleEngine(ocfg)
    restart.load(o, path)
    for a, b in zip(g.download_flow(), o.download_flow()):
        assert np.array_equal(a, b)
    for s in range(2):
        pa, pb = g.download_particles(s), o.download_particles(s)
        for k in ("ids", "diam", "x", "y", "z", "u", "v", "w"):
            assert np.array_equal(pa[k], pb[k]), (s, k)
    # and back: the oracle's file into a fresh CUDA handle
    path2 = str(tmp_path / "restart.h5.back")
    restart.save(o, path2)
    g2 = Engine(cfg)
    restart.load(g2, path2)
    for a, b in zip(g.download_flow(), g2.download_flow()):
        assert np.array_equal(a, b)
    for e in (g, g2, o):
        e.close()


def test_gpu_restart_load_coarse(tmp_path):
    c = OracleEngine(make_config(32, mode=_abi.MODE_FLOW))
    rng = np.random.default_rng(2)
    fields = [rng.standard_normal((32, 32, 32)) for _ in range(4)]
    c.upload_flow(*fields)
    path = str(tmp_path / "coarse.h5")
    restart.save(c, path)
    g, o = Engine(make_config(64, mode=_abi.MODE_FLOW)), OracleEngine(make_config(64, mode=_abi.MODE_FLOW))
    restart.load_coarse(g, path)
    o.upload_flow_coarse(*fields)
    for a, b in zip(g.download_flow(), o.download_flow()):
        assert np.array_equal(a, b)
    for e in (g, o, c):
        e.close()
