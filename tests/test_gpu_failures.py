"""Failure paths of the CUDA library, made without faulting the GPU.

- A NaN cell uploaded from the host: Julia's maximum(abs, U) propagates it
  (src/flows/timestep.jl:48-64), the time step is NaN and the call returns
  LCS_ENONFINITE, launch by launch and inside the step graphs alike.
- The bounded device waits: the test hook lcs_debug_unreachable_waits makes
  one kind of wait unreachable (a grid-barrier arrival that never comes, or
  TMA plane barriers expecting 16 bytes more than the copies deliver).  The
  wait runs out at its bound, the call returns LCS_ETIMEDOUT, and the GPU
  context stays usable: a new handle afterwards equals the oracle.
"""

import ctypes as C

import numpy as np
import pytest

from helpers import make_config
from lcs_b200 import Engine, LCSError, inits
from lcs_b200 import _abi as F
from oracle_engine import OracleEngine

pytestmark = pytest.mark.gpu


def flow_with(n, value, where=(5, 6, 7), field=1):
    U, V, W, P = inits.spectral_flow(n, seed=2)
    (U, V, W)[field][where] = value
    return U, V, W, P


@pytest.mark.parametrize("precision", [F.PRECISION_FP64, F.PRECISION_FP32_MIXED])
@pytest.mark.parametrize("graphs", [0, 1])
def test_nan_cell_gives_enonfinite(graphs, precision):
    cfg = make_config(32, Re=100.0, itrmax=12, graphs=graphs, precision=precision,
                      forcing=F.FORCING_LINEAR_POWER, power=0.5, species=[{"n": 500, "density_ratio": 843.0}])
    e = Engine(cfg)
    e.upload_flow(*flow_with(32, np.nan))
    x, y, z = inits.random_positions(500, 4)
    zero = np.zeros(500)
    e.upload_particles(0, np.full(500, 0.02), x, y, z, zero, zero, zero)
    assert np.isnan(e.flow_timestep())
    with pytest.raises(LCSError) as ei:
        if graphs:
            e.step(1)
        else:
            e.timestep()
    assert ei.value.code == F.ENONFINITE
    e.close()


def test_nan_agrees_with_the_oracle():
    cfg = make_config(16, mode=F.MODE_FLOW, Re=50.0)
    flow = flow_with(16, np.nan, where=(1, 2, 3), field=2)
    for cls in (Engine, OracleEngine):
        e = cls(cfg)
        e.upload_flow(*flow)
        assert np.isnan(e.flow_timestep())
        e.close()


def couple_cfg(precision=F.PRECISION_FP64):
    return make_config(32, mode=F.MODE_FLOW, Re=100.0, itrmin=6, itrmax=9, epsp=1e-30, precision=precision)


def run_couple(cls, cfg, flow):
    e = cls(cfg)
    e.upload_flow(*flow)
    lg = e.couple(2, 0.004)
    out = e.download_flow()
    e.close()
    return lg, out


@pytest.mark.parametrize("kind,precision", [(1, F.PRECISION_FP64), (2, F.PRECISION_FP64),
                                            (2, F.PRECISION_FP32_MIXED)])
def test_unreachable_wait_returns_etimedout(kind, precision):
    """kind 1: the face kernel's grid barrier (overlap sweeps); kind 2: the
    row-warp sweep's TMA plane barriers."""
    cfg = couple_cfg(precision)
    flow = inits.spectral_flow(32, seed=5)
    e = Engine(cfg)
    e.upload_flow(*flow)
    assert e.lib.lcs_debug_unreachable_waits(e.handle, kind) == 0
    with pytest.raises(LCSError) as ei:
        e.couple(2, 0.004)
    assert ei.value.code == F.ETIMEDOUT
    assert e.lib.lcs_debug_unreachable_waits(e.handle, 0) == 0
    with pytest.raises(LCSError) as ei:  # the wait error is sticky for the handle
        e.couple(2, 0.004)
    assert ei.value.code == F.ETIMEDOUT
    e.close()
    # the context is intact: a new handle computes what the oracle computes
    if precision == F.PRECISION_FP64:
        (lg, fg), (lo, fo) = run_couple(Engine, cfg, flow), run_couple(OracleEngine, cfg, flow)
        assert lg["itr"] == lo["itr"] and lg["sweeps"] == lo["sweeps"]
        for a, b in zip(fg, fo):
            assert np.array_equal(a, b)
    else:
        lg, _ = run_couple(Engine, cfg, flow)
        assert lg["sweeps"] == 9


def test_unreachable_wait_inside_the_step_graph():
    cfg = make_config(32, Re=100.0, itrmin=6, itrmax=9, epsp=1e-30, graphs=1, forcing=F.FORCING_LINEAR_POWER,
                      power=0.5, species=[{"n": 500, "density_ratio": 843.0}])
    e = Engine(cfg)
    e.upload_flow(*inits.spectral_flow(32, seed=6))
    x, y, z = inits.random_positions(500, 4)
    zero = np.zeros(500)
    e.upload_particles(0, np.full(500, 0.02), x, y, z, zero, zero, zero)
    e.step(1)
    assert e.lib.lcs_debug_unreachable_waits(e.handle, 1) == 0
    with pytest.raises(LCSError) as ei:
        e.step(2)
    assert ei.value.code == F.ETIMEDOUT
    e.close()


def test_debug_hook_rejects_unknown_kinds():
    e = Engine(couple_cfg())
    assert e.lib.lcs_debug_unreachable_waits(e.handle, 3) == F.EINVAL
    assert e.lib.lcs_debug_unreachable_waits(e.handle, -1) == F.EINVAL
    e.close()
    assert C.c_int(F.ETIMEDOUT).value < 0
