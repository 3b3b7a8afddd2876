"""The `upsample` init (src/LCSIO/upsample.jl:1-91) on the device against the
oracle: bit-exact in FP64; in the FP32-mixed form each fine value is the FP64
value rounded once to FP32.  Steps after an upsampled init follow the oracle
within the north-star field tolerance."""

import numpy as np
import pytest

from helpers import make_config, rel_l2
from lcs_b200 import Engine, _abi
from oracle_engine import OracleEngine

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims", [(32, 32, 32), (48, 32, 40), (128, 128, 128)])
def test_upsample_equals_oracle(dims):
    cfg = make_config(dims=dims, mode=_abi.MODE_FLOW)
    g, o = Engine(cfg), OracleEngine(cfg)
    rng = np.random.default_rng(dims[0])
    coarse = [rng.standard_normal((dims[2] // 2, dims[1] // 2, dims[0] // 2)) for _ in range(4)]
    for e in (g, o):
        e.upload_flow_coarse(*coarse)
    for a, b in zip(g.download_flow(), o.download_flow()):
        assert np.array_equal(a, b)
    g.close()
    o.close()


def test_upsample_fp32_form_rounds_once():
    dims = (32, 32, 32)
    o = OracleEngine(make_config(dims=dims, mode=_abi.MODE_FLOW))
    g = Engine(make_config(dims=dims, mode=_abi.MODE_FLOW, precision=_abi.PRECISION_FP32_MIXED))
    rng = np.random.default_rng(1)
    coarse = [rng.standard_normal((16, 16, 16)) for _ in range(4)]
    for e in (g, o):
        e.upload_flow_coarse(*coarse)
    for a, b in zip(g.download_flow(), o.download_flow()):
        assert np.array_equal(a, b.astype(np.float32).astype(np.float64))
    g.close()
    o.close()


def test_steps_after_upsample_follow_oracle():
    n = 32
    cfg = make_config(n, mode=_abi.MODE_FLOW, Re=100.0, forcing=_abi.FORCING_LINEAR_POWER, power=0.5)
    g, o = Engine(cfg), OracleEngine(cfg)
    rng = np.random.default_rng(3)
    coarse = [rng.standard_normal((n // 2,) * 3) * 0.3 for _ in range(3)] + [np.zeros((n // 2,) * 3)]
    for e in (g, o):
        e.upload_flow_coarse(*coarse)
    for e in (g, o):
        e.step(3)
    for a, b in zip(g.download_flow(), o.download_flow()):
        assert rel_l2(a, b) <= 1e-10
    g.close()
    o.close()
