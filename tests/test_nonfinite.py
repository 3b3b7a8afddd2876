"""Non-finite fields on the oracle: Julia's maximum(abs, U) and min(cands...)
propagate a NaN (src/flows/timestep.jl:48-64), so a NaN cell gives a NaN dt
and the C ABI reports LCS_ENONFINITE instead of stepping on."""

import ctypes as C
import math

import numpy as np
import pytest

from helpers import make_config
from lcs_b200 import LCSError, inits
from lcs_b200 import _abi as F
from oracle_engine import OracleEngine, load_oracle


def nan_flow(n, where=(3, 4, 5), field=0, value=np.nan):
    U, V, W, P = inits.spectral_flow(n, seed=1)
    (U, V, W)[field][where] = value
    return U, V, W, P


@pytest.mark.parametrize("field", [0, 1, 2])
def test_nan_cell_gives_nan_dt_and_enonfinite(field):
    e = OracleEngine(make_config(16, mode=F.MODE_FLOW, Re=50.0))
    e.upload_flow(*nan_flow(16, field=field))
    assert math.isnan(e.flow_timestep())
    with pytest.raises(LCSError) as ei:
        e.timestep()
    assert ei.value.code == F.ENONFINITE
    e.close()


def test_nan_diameter_gives_enonfinite():
    """particles/timestep.jl: maximum(diams) propagates a NaN diameter too."""
    e = OracleEngine(make_config(16, Re=50.0, species=[{"n": 50, "density_ratio": 843.0}]))
    e.upload_flow(*inits.spectral_flow(16, seed=1))
    x, y, z = inits.random_positions(50, 3)
    d = np.full(50, 0.01)
    d[7] = np.nan
    zero = np.zeros(50)
    e.upload_particles(0, d, x, y, z, zero, zero, zero)
    assert math.isnan(e.particles_timestep())
    with pytest.raises(LCSError) as ei:
        e.timestep()
    assert ei.value.code == F.ENONFINITE
    e.close()


def test_infinite_cell_gives_zero_dt_limit():
    """An infinite velocity gives cfl*dx/Inf = 0: dt is not positive."""
    e = OracleEngine(make_config(16, mode=F.MODE_FLOW, Re=50.0))
    e.upload_flow(*nan_flow(16, value=np.inf))
    assert e.flow_timestep() == 0.0
    with pytest.raises(LCSError) as ei:
        e.timestep()
    assert ei.value.code == F.ENONFINITE
    e.close()


def test_noalloc_restatement_propagates_nan():
    lib = load_oracle()
    n, h = 16, 3
    U, V, W, _ = nan_flow(n, field=1)
    arrs = []
    for a in (U, V, W):
        b = np.zeros((n + 2 * h,) * 3)
        b[h:h + n, h:h + n, h:h + n] = a
        arrs.append(b)
    out = C.c_double()
    rc = lib.lcs_flow_timestep_noalloc(*(a.ctypes.data_as(C.c_void_p) for a in arrs), (C.c_int32 * 3)(n, n, n), h,
                                       0.3, 1.0, 50.0, C.byref(out), None)
    assert rc == 0 and math.isnan(out.value)
