"""Device statistics (lcs_flow_stat, `Flows.stat` of src/flows/stat.jl:66-153)
against the oracle's and against the host restatement, in both precision forms.
Means are summed in different orders: agreement to 1e-12 relative; max/min are
exact.  The call changes no state."""

import math

import numpy as np
import pytest

from helpers import make_config
from lcs_b200 import Engine, _abi, inits, stats
from oracle_engine import OracleEngine

pytestmark = pytest.mark.gpu
KEYS = ("urms", "k", "epsilon", "tau_eta", "l_mu", "l_eta", "Re_lambda", "k_eta", "skewness", "flatness")


@pytest.mark.parametrize("n", [32, 48])
def test_device_flow_stat_equals_oracle(n):
    nu = 0.005
    cfg = make_config(n, mode=_abi.MODE_FLOW, Re=1.0 / nu)
    g, o = Engine(cfg), OracleEngine(cfg)
    U, V, W, P = inits.spectral_flow(n, seed=n)
    for e in (g, o):
        e.upload_flow(U, V, W, P)
    before = g.download_flow()
    a, b = g.flow_stat(), o.flow_stat()
    for k in KEYS + ("u_mean", "v_mean", "w_mean"):
        assert math.isclose(a[k], b[k], rel_tol=1e-12, abs_tol=1e-15), (k, a[k], b[k])
    for k in ("u_max", "v_max", "w_max", "u_min", "v_min", "w_min"):
        assert a[k] == b[k]
    for x, y in zip(g.download_flow(), before):
        assert np.array_equal(x, y)


def test_device_flow_stat_fp32_form():
    n, nu = 32, 0.01
    e = Engine(make_config(n, mode=_abi.MODE_FLOW, Re=1.0 / nu, precision=_abi.PRECISION_FP32_MIXED))
    U, V, W, P = inits.spectral_flow(n, seed=5)
    e.upload_flow(U, V, W, P)
    Uf, Vf, Wf, _ = e.download_flow()  # the FP32 values the device holds
    got, ref = e.flow_stat(), stats.flow_stat(Uf, Vf, Wf, nu)
    for k in KEYS:
        assert math.isclose(got[k], ref[k], rel_tol=1e-12), (k, got[k], ref[k])


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_FP32_MIXED])
def test_device_divergence_equals_oracle(precision):
    n = 48
    cfg = make_config(n, mode=_abi.MODE_FLOW)
    g = Engine(make_config(n, mode=_abi.MODE_FLOW, precision=precision))
    o = OracleEngine(cfg)
    U, V, W, P = inits.spectral_flow(n, seed=9)
    rng = np.random.default_rng(3)
    U = U + 1e-3 * rng.standard_normal(U.shape)  # not divergence-free
    g.upload_flow(U, V, W, P)
    o.upload_flow(*g.download_flow())  # the values the device holds (FP32-rounded in that form)
    (ra, ma), (rb, mb) = g.flow_divergence(), o.flow_divergence()
    assert math.isclose(ra, rb, rel_tol=1e-12), (ra, rb)
    if precision == _abi.PRECISION_FP64:
        assert ma == mb
    else:  # the FP32 form's object code may fuse the FP64 multiply-adds
        assert math.isclose(ma, mb, rel_tol=1e-12)
    g.close()
    o.close()
