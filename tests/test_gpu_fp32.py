"""The FP32-mixed form against the plain FP64 form, on identical seeded inputs.

FP32-mixed keeps fields, stencils, HSMAC sweeps and the fluid velocity that
particles see in FP32; the HSMAC residual and exit test, the forcing's energy
reductions, the time step and the particle state stay FP64.  Its results are
not bit-comparable with FP64, so each test states its tolerance:
- a round trip through the device rounds every value to the nearest FP32;
- one couple of 20 sweeps: rel-L2 <= 1e-5 for U, V, W (FP32 unit roundoff is
  6e-8; the sweeps accumulate it; measured 1.2e-7) and the two FP32 sweep
  kernels agree to 2e-6 (they contract multiply-adds differently); P, a sum of
  increments dp/dt that largely cancel, to 1e-3 (measured 2e-5);
- ten full steps with forcing and particles: rel-L2 <= 1e-4 for U, V, W (the
  bound stated for the precision form; measured 4.4e-7) and <= 1e-3 for
  P, particle positions <= 1e-6 and velocities <= 1e-4.
"""

import numpy as np
import pytest

from helpers import make_config, rel_l2
from lcs_b200 import Engine, _abi, inits

F = _abi
pytestmark = pytest.mark.gpu


def fp32_cfg(*args, **kw):
    return make_config(*args, precision=F.PRECISION_FP32_MIXED, **kw)


def test_fp32_round_trip_rounds_to_nearest_float():
    e = Engine(fp32_cfg(24, mode=F.MODE_FLOW))
    rng = np.random.default_rng(1)
    U, V, W, P = (rng.standard_normal(e.interior_shape) for _ in range(4))
    e.upload_flow(U, V, W, P)
    for a, b in zip(e.download_flow(), (U, V, W, P)):
        assert np.array_equal(a, b.astype(np.float32).astype(np.float64))
    e.close()


@pytest.mark.parametrize("tb,ov", [(True, True), (True, False), (False, True), (False, False)])
def test_fp32_couple_close_to_fp64(tb, ov, monkeypatch):
    U, V, W, P = inits.spectral_flow(64, seed=5)
    out = {}
    for name, prec, sweep in (("fp64", F.PRECISION_FP64, "rw"), ("fp32", F.PRECISION_FP32_MIXED, "rw"),
                              ("fp32-plain", F.PRECISION_FP32_MIXED, "plain")):
        monkeypatch.setenv("LCS_B200_FUSED_SWEEP", sweep)
        e = Engine(make_config(64, mode=F.MODE_FLOW, time_blocking=tb, overlap=ov, itrmin=6, itrmax=20, epsp=1e-12,
                               precision=prec))
        e.upload_flow(U, V, W, P)
        lg = e.couple(2, 0.004)
        out[name] = (lg, e.download_flow())
        e.close()
    l64, f64 = out["fp64"]
    l32, f32 = out["fp32"]
    lp, fp = out["fp32-plain"]
    assert l32["sweeps"] == l64["sweeps"] == lp["sweeps"]
    assert abs(l32["div"] - l64["div"]) <= 1e-3 * l64["div"]
    names = ("U", "V", "W", "P")
    errs64 = [rel_l2(a, b) for a, b in zip(f32, f64)]
    errsp = [rel_l2(a, b) for a, b in zip(f32, fp)]
    print("fp32 vs fp64", dict(zip(names, errs64)), "rw vs plain", dict(zip(names, errsp)))
    assert max(errs64[:3]) <= 1e-5, errs64
    assert max(errsp[:3]) <= 2e-6, errsp
    # P sums 20 increments dp/dt that largely cancel: its relative error is larger
    assert errs64[3] <= 1e-3 and errsp[3] <= 1e-3, (errs64, errsp)


@pytest.mark.parametrize("variant", ["8", "5"])
def test_fp32_row_warp_variants_agree(variant, monkeypatch):
    U, V, W, P = inits.spectral_flow(96, seed=6)
    out = []
    for v in (variant, "13"):
        monkeypatch.setenv("LCS_B200_RW", v)
        e = Engine(fp32_cfg(96, mode=F.MODE_FLOW, itrmin=6, itrmax=9, epsp=1e-12))
        e.upload_flow(U, V, W, P)
        e.couple(2, 0.003)
        out.append(e.download_flow())
        e.close()
    errs = [rel_l2(a, b) for a, b in zip(*out)]
    assert max(errs[:3]) <= 2e-6 and errs[3] <= 1e-3, errs


@pytest.mark.parametrize("forcing", [F.FORCING_LINEAR_POWER, F.FORCING_RC_ENERGY])
def test_fp32_ten_steps_close_to_fp64(forcing):
    n, npart = 32, 3000
    U, V, W, P = inits.spectral_flow(n, seed=7)
    species = [{"n": npart, "density_ratio": 843.0}, {"n": npart, "density_ratio": 843.0}]
    res = {}
    for prec in (F.PRECISION_FP64, F.PRECISION_FP32_MIXED):
        cfg = make_config(n, forcing=forcing, power=0.5, energy=0.649, kmin=1, kmax=2, coarse=8, Re=100.0,
                          itrmin=6, itrmax=30, epsp=1e-8, species=species, graphs=1, precision=prec)
        e = Engine(cfg)
        e.upload_flow(U, V, W, P)
        for s in range(2):
            x, y, z = inits.random_positions(npart, 10 + s)
            zero = np.zeros(npart)
            e.upload_particles(s, np.full(npart, 0.02 * (1 + s)), x, y, z, zero, zero, zero)
            e.init_particle_velocity(s)
        e.step(10)
        res[prec] = (e.download_flow(), [e.download_particles(s) for s in range(2)])
        e.close()
    (f64, p64), (f32, p32) = res[F.PRECISION_FP64], res[F.PRECISION_FP32_MIXED]
    errs = [rel_l2(a, b) for a, b in zip(f32, f64)]
    perrs = [{k: rel_l2(a[k], b[k]) for k in ("x", "y", "z", "u", "v", "w")} for a, b in zip(p32, p64)]
    print("fields", errs, "particles", perrs)
    assert max(errs[:3]) <= 1e-4, errs
    assert errs[3] <= 1e-3, errs
    for pe in perrs:
        assert max(pe[k] for k in ("x", "y", "z")) <= 1e-6, pe
        assert max(pe[k] for k in ("u", "v", "w")) <= 1e-4, pe


@pytest.mark.parametrize("dims,tb,ov", [((64, 64, 64), True, True), ((64, 64, 64), False, False),
                                        ((200, 48, 40), True, True), ((136, 40, 24), False, True),
                                        ((40, 24, 32), True, False)])
def test_fp32_two_row_warps_agree_with_one_row_warps(dims, tb, ov, monkeypatch):
    """The FP32 default tiles (29 rows, two rows per warp: LCS_B200_RW=29)
    against 13-row tiles of one row per warp, on grids with several tile
    columns, partial tiles and few z planes: the same arithmetic per cell, so
    U, V, W agree to 2e-6 and P to 1e-3 after a couple of 12 sweeps (measured
    values printed)."""
    rng = np.random.default_rng(sum(dims))
    flow = [rng.standard_normal((dims[2], dims[1], dims[0])) * 0.5 for _ in range(3)] + \
        [rng.standard_normal((dims[2], dims[1], dims[0])) * 0.1]
    out = {}
    for rows in ("29", "13"):
        monkeypatch.setenv("LCS_B200_RW", rows)
        e = Engine(fp32_cfg(dims=dims, mode=F.MODE_FLOW, time_blocking=tb, overlap=ov, itrmin=6, itrmax=12,
                            epsp=1e-12))
        e.upload_flow(*flow)
        lg = e.couple(2, 0.003)
        out[rows] = (lg, e.download_flow())
        e.close()
    (l2, f2), (l1, f1) = out["29"], out["13"]
    assert l2["sweeps"] == l1["sweeps"]
    errs = [rel_l2(a, b) for a, b in zip(f2, f1)]
    same = [bool(np.array_equal(a, b)) for a, b in zip(f2, f1)]
    print("29-row vs 13-row", errs, "bitwise", same)
    assert max(errs[:3]) <= 2e-6, errs
    assert errs[3] <= 1e-3, errs
    assert abs(l2["div"] - l1["div"]) <= 1e-4 * abs(l1["div"])
