"""Host statistics (the restated `Flows.stat`, src/flows/stat.jl:66-153, and
E(k)) on fields with analytic answers."""

import math

import numpy as np

from lcs_b200 import stats


def grid(n):
    x = (np.arange(n) + 0.5) * 2 * math.pi / n
    return np.meshgrid(x, x, x, indexing="ij")  # [k, j, i] order: z, y, x


def test_shear_mode_urms_and_dissipation():
    n, nu = 32, 0.01
    z, y, x = grid(n)
    U = np.sin(y)
    V = np.zeros_like(U)
    W = np.zeros_like(U)
    st = stats.flow_stat(U, V, W, nu)
    assert math.isclose(st["urms"], math.sqrt(0.5 / 3), rel_tol=1e-12)
    assert math.isclose(st["k"], 0.25, rel_tol=1e-12)
    # s12 = cos(y)/2 up to the o4 stencil error (~(dx^4) k^4 * 3/640): s2 = 4 <s12^2> = 1/2
    assert math.isclose(st["epsilon"], 0.5 * nu, rel_tol=1e-4)


def test_energy_spectrum_of_single_modes():
    n = 32
    z, y, x = grid(n)
    U = np.cos(3 * x)          # energy <u^2>/2 = 1/4 at |k| = 3
    V = 2.0 * np.sin(5 * z)    # energy 1 at |k| = 5
    W = np.zeros_like(U)
    e = stats.energy_spectrum(U, V, W)
    assert math.isclose(e[3], 0.25, rel_tol=1e-12)
    assert math.isclose(e[5], 1.0, rel_tol=1e-12)
    assert math.isclose(e.sum(), 1.25, rel_tol=1e-12)
    # Parseval: sum of E(k) = <|u|^2> / 2
    assert math.isclose(e.sum(), 0.5 * float(np.mean(U ** 2 + V ** 2 + W ** 2)), rel_tol=1e-12)


def test_particle_rms():
    u = np.array([1.0, -1.0]); v = np.zeros(2); w = np.zeros(2)
    assert math.isclose(stats.particle_rms_velocity(u, v, w), math.sqrt(1 / 3), rel_tol=1e-15)


KEYS = ("urms", "k", "epsilon", "tau_eta", "l_mu", "l_eta", "Re_lambda", "k_eta", "skewness", "flatness")


def test_oracle_flow_stat_equals_host_restatement():
    """The oracle's lcs_flow_stat (C, sums in i, j, k order) against the numpy
    restatement (pairwise sums): the same means to rounding."""
    from helpers import make_config
    from lcs_b200 import _abi, inits
    from oracle_engine import OracleEngine

    n, nu = 24, 0.01
    e = OracleEngine(make_config(n, mode=_abi.MODE_FLOW, Re=1.0 / nu))
    U, V, W, P = inits.spectral_flow(n, seed=3)
    e.upload_flow(U, V, W, P)
    got = e.flow_stat()
    ref = stats.flow_stat(U, V, W, nu)
    for k in KEYS:
        assert math.isclose(got[k], ref[k], rel_tol=1e-12), (k, got[k], ref[k])
    for c, a in zip("uvw", (U, V, W)):
        assert math.isclose(got[c + "_mean"], float(a.mean()), rel_tol=1e-9, abs_tol=1e-15)
        assert got[c + "_max"] == float(a.max()) and got[c + "_min"] == float(a.min())
    assert got["L"] == 0.0 and got["C_epsilon"] == 0.0
    e.close()


def test_oracle_divergence_of_known_fields():
    """lcs_flow_divergence on the oracle: zero for fields independent of their
    own axis, and the restated HSMAC difference for a cosine (periodic)."""
    from helpers import make_config
    from lcs_b200 import _abi
    from oracle_engine import OracleEngine

    n = 16
    e = OracleEngine(make_config(n, mode=_abi.MODE_FLOW))
    z, y, x = np.meshgrid(*[np.arange(1, n + 1)] * 3, indexing="ij")
    e.upload_flow(np.sin(y * 0.3), np.cos(z * 0.7), np.sin(x * 1.1), np.zeros((n, n, n)))
    rms, mx = e.flow_divergence()
    assert rms == 0.0 and mx == 0.0
    U = np.cos(2 * np.pi * x / n)
    e.upload_flow(U, np.zeros_like(U), np.zeros_like(U), np.zeros_like(U))
    dxi = n / (2 * np.pi)
    div = dxi * (-np.roll(U, 1, axis=2) + U)
    rms, mx = e.flow_divergence()
    assert math.isclose(rms, math.sqrt(np.mean(div ** 2)), rel_tol=1e-13)
    assert mx == np.abs(div).max()
    e.close()
