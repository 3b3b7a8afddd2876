"""The `upsample` init (src/LCSIO/upsample.jl:1-91) on the oracle against a
numpy restatement of trilinear_upsample2x! (periodic one-cell halo, sums left
to right as written there): bit-exact."""

import numpy as np
import pytest

from helpers import make_config
from lcs_b200 import _abi
from oracle_engine import OracleEngine


def upsample_numpy(c):
    """c is [k, j, i]; returns the fine [2k, 2j, 2i] interior."""
    s = lambda di=0, dj=0, dk=0: np.roll(c, (-dk, -dj, -di), axis=(0, 1, 2))  # noqa: E731
    c000, c100, c010, c001 = c, s(1), s(0, 1), s(0, 0, 1)
    c110, c101, c011, c111 = s(1, 1), s(1, 0, 1), s(0, 1, 1), s(1, 1, 1)
    nz, ny, nx = c.shape
    f = np.empty((2 * nz, 2 * ny, 2 * nx))
    f[0::2, 0::2, 0::2] = c000
    f[0::2, 0::2, 1::2] = (1 / 2) * (c000 + c100)
    f[0::2, 1::2, 0::2] = (1 / 2) * (c000 + c010)
    f[1::2, 0::2, 0::2] = (1 / 2) * (c000 + c001)
    f[0::2, 1::2, 1::2] = (1 / 4) * (((c000 + c100) + c010) + c110)
    f[1::2, 0::2, 1::2] = (1 / 4) * (((c000 + c100) + c001) + c101)
    f[1::2, 1::2, 0::2] = (1 / 4) * (((c000 + c010) + c001) + c011)
    f[1::2, 1::2, 1::2] = (1 / 8) * (((((((c000 + c100) + c010) + c001) + c110) + c101) + c011) + c111)
    return f


@pytest.mark.parametrize("dims", [(16, 16, 16), (24, 16, 20)])
def test_oracle_upsample_equals_numpy(dims):
    cfg = make_config(dims=dims, mode=_abi.MODE_FLOW)
    e = OracleEngine(cfg)
    rng = np.random.default_rng(4)
    coarse = [rng.standard_normal((dims[2] // 2, dims[1] // 2, dims[0] // 2)) for _ in range(4)]
    e.upload_flow_coarse(*coarse)
    for got, c in zip(e.download_flow(), coarse):
        assert np.array_equal(got, upsample_numpy(c))
    e.close()


def test_upsample_of_a_constant_and_a_mode():
    n = 16
    e = OracleEngine(make_config(n, mode=_abi.MODE_FLOW))
    m = n // 2
    x = np.arange(m) * (2 * np.pi / m)
    wave = np.broadcast_to(np.cos(x)[None, None, :], (m, m, m)).copy()
    e.upload_flow_coarse(np.full((m, m, m), 0.75), wave, np.zeros((m, m, m)), np.full((m, m, m), -2.0))
    U, V, W, P = e.download_flow()
    assert np.all(U == 0.75) and np.all(W == 0.0) and np.all(P == -2.0)
    # midpoints of a cosine: the average of its two coarse neighbours, periodic
    assert np.allclose(V[..., 1::2], 0.5 * (np.cos(x) + np.cos(np.roll(x, -1))), rtol=0, atol=1e-15)
    e.close()
