"""Pins of the CPU oracle against the reference's own deterministic test
assertions (tests/golden/known_answers.json, extracted from the reference's
test files by tests/golden/make_known_answers.py)."""

import ctypes as C
import json
import math
import os

import numpy as np
import pytest

from helpers import make_config
from lcs_b200 import _abi
from oracle_engine import OracleEngine, load_oracle

KA = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))


def dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def test_kcount():  # lib/fouriertools/test/runtests.jl:86-87
    lib = load_oracle()
    assert lib.lcs_oracle_kcount(1) == KA["kcount"]["1"] == 18
    assert lib.lcs_oracle_kcount(2) == KA["kcount"]["2"] == 62


def test_kset1_and_canonical_form():  # runtests.jl:71-83, 62-69
    lib = load_oracle()
    buf = (C.c_int32 * 384)()
    n = lib.lcs_oracle_kset(1, buf, 128)
    got = {tuple(buf[3 * q:3 * q + 3]) for q in range(n)}
    assert got == {tuple(v) for v in KA["kset1"]["set"]}
    assert n == KA["kcount"]["1"] // 2
    # every generated vector is canonical: first non-zero component positive
    for K in (1, 2, 3):
        n = lib.lcs_oracle_kset(K, buf, 128)
        assert n == lib.lcs_oracle_kcount(K) // 2
        for q in range(n):
            v = buf[3 * q:3 * q + 3]
            first = next(x for x in v if x != 0)
            assert first > 0
    for case in KA["canon"]:
        v = case["in"]
        first = next((x for x in v if x != 0), 0)
        canon = [-x for x in v] if first < 0 else v
        assert canon == case["out"]


def test_enespe_constant_spectrum():  # runtests.jl:92-96
    lib = load_oracle()
    val = float(KA["enespe_constant"]["value"])
    for kmax in (1, 2):
        nm = (kmax + 1) * (2 * kmax + 1) ** 2
        hat = np.zeros((3, nm, 2))
        hat[:, :, 0] = val
        norm = 16.0 ** 3
        for k0 in range(1, kmax + 1):
            e = lib.lcs_oracle_enespe(dp(hat), kmax, k0, norm)
            assert e == lib.lcs_oracle_kcount(k0) * 3 / 2


def sincospi(x):
    s, c = C.c_double(), C.c_double()
    load_oracle().lcs_oracle_sincospi(x, C.byref(s), C.byref(c))
    return complex(c.value, s.value)


def test_sirdft_equals_masked_inverse_dft():  # runtests.jl:99-127
    lib = load_oracle()
    prop = KA["sirdft_property"]
    n, kmin, kmax = prop["n"], prop["kmin"], prop["kmax"]
    rng = np.random.default_rng(7)
    A = rng.random((n, n, n))  # [z, y, x]
    A_hat = np.fft.rfftn(A)    # [kz, ky, kx], kx in 0..n/2
    KX, KY = kmax + 1, 2 * kmax + 1
    crop = np.zeros((KY, KY, KX, 2))
    masked = np.zeros_like(A_hat)
    for kz in range(-kmax, kmax + 1):
        for ky in range(-kmax, kmax + 1):
            for kx in range(0, kmax + 1):
                c = A_hat[kz % n, ky % n, kx] / n ** 3
                crop[kz + kmax, ky + kmax, kx] = (c.real, c.imag)
                if kmin - 0.5 <= math.sqrt(kx * kx + ky * ky + kz * kz) < kmax + 0.5:
                    masked[kz % n, ky % n, kx] = A_hat[kz % n, ky % n, kx]
    A3 = np.fft.irfftn(masked, s=(n, n, n), axes=(0, 1, 2))
    crop = np.ascontiguousarray(crop)
    A2 = np.zeros((n, n, n))
    for k in range(n):
        ek = sincospi(2 * k / n)
        for j in range(n):
            ej = sincospi(2 * j / n)
            for i in range(n):
                ei = sincospi(2 * i / n)
                A2[k, j, i] = lib.lcs_oracle_sirdft(dp(crop), kmin, kmax, ei.real, ei.imag, ej.real, ej.imag,
                                                    ek.real, ek.imag)
    np.testing.assert_allclose(A2, A3, rtol=1e-12, atol=1e-13)


def test_sincospi_exact_points():
    assert sincospi(0.0) == 1 + 0j
    assert sincospi(0.5) == 0 + 1j
    assert sincospi(1.0) == -1 + 0j
    assert sincospi(-0.5) == 0 - 1j
    for x in np.linspace(-3, 3, 97):
        z = sincospi(float(x))
        r = math.fmod(float(x), 2.0)
        assert abs(z - complex(math.cos(math.pi * r), math.sin(math.pi * r))) < 1e-15


def test_boxmean_piecewise_constant_is_exact():  # test/test_flows.jl:122-136
    lib = load_oracle()
    b = KA["boxmean"]
    n, c, h = b["dims"][0], b["coarse_dims"][0], b["halo_size"]
    f = n // c
    ref = np.arange(1, c ** 3 + 1, dtype=np.float64).reshape(c, c, c)  # [kc, jc, ic]: x fastest like reshape(1:8,2,2,2)
    A = np.zeros((n + 2 * h,) * 3)
    A[h:h + n, h:h + n, h:h + n] = np.repeat(np.repeat(np.repeat(ref, f, 0), f, 1), f, 2)
    out = np.zeros(c ** 3)
    lib.lcs_oracle_boxmean(dp(A), n, h, c, dp(out))
    assert np.array_equal(out.reshape(c, c, c), ref)


def test_rcf_helpers():  # test/test_flows.jl:138-148
    r = KA["rcf_helpers"]
    assert load_oracle().lcs_oracle_phase_shift(r["grid"][0], r["coarse_size"]) == r["phase_shift"]
    assert r["grid"][0] // r["coarse_size"] == r["filter_size"]


@pytest.mark.parametrize("coloring", [_abi.COLORING_RED_BLACK, _abi.COLORING_RED_BLACK_FAST])
def test_coloring_reference_masks(coloring):  # lib/parallel/test/runtests.jl:73-113
    lib = load_oracle()
    lo = (C.c_int32 * 3)(2, 2, 2)
    hi = (C.c_int32 * 3)(4, 4, 4)
    for color, key in ((0, "ref0x00"), (1, "ref0x01")):
        m = (C.c_int32 * 27)()
        lib.lcs_oracle_color_mask(coloring, 0, lo, hi, color, m)
        got = np.zeros((5, 5, 5), dtype=int)  # [i, j, k] 1-based 1..5 -> 0..4
        arr = np.array(m[:]).reshape(3, 3, 3)  # [k, j, i]
        for k in range(3):
            for j in range(3):
                for i in range(3):
                    got[1 + i, 1 + j, 1 + k] = arr[k, j, i]
        assert np.array_equal(got, np.array(KA[key]["array"]))


@pytest.mark.parametrize("coloring,block", [(_abi.COLORING_RED_BLACK, 0), (_abi.COLORING_RED_BLACK_FAST, 0),
                                            (_abi.COLORING_RED_BLACK_BLOCK, 2)])
@pytest.mark.parametrize("lo,hi", [((2, 2, 2), (4, 4, 4)), ((1, 1, 1), (4, 4, 4))])
def test_coloring_covers_axes_once(coloring, block, lo, hi):  # runtests.jl:48-71
    lib = load_oracle()
    n = hi[0] - lo[0] + 1
    tot = np.zeros(n ** 3, dtype=int)
    for color in (0, 1):
        m = (C.c_int32 * n ** 3)()
        lib.lcs_oracle_color_mask(coloring, block, (C.c_int32 * 3)(*lo), (C.c_int32 * 3)(*hi), color, m)
        tot += np.array(m[:])
    assert np.all(tot == 1)


def test_red_black_skips_negative_odd_sums():
    """RedBlack tests `sum(i) % 0x02 == color` with Julia's signed `%`: cells with
    a negative odd index sum belong to neither colour (foraxes.jl:82-88)."""
    lib = load_oracle()
    lo, hi = (-1, -1, -1), (1, 1, 1)
    seen = np.zeros(27, dtype=int)
    for color in (0, 1):
        m = (C.c_int32 * 27)()
        lib.lcs_oracle_color_mask(_abi.COLORING_RED_BLACK, 0, (C.c_int32 * 3)(*lo), (C.c_int32 * 3)(*hi), color, m)
        seen += np.array(m[:])
    idx = np.array([(i + j + k) for k in (-1, 0, 1) for j in (-1, 0, 1) for i in (-1, 0, 1)])
    assert np.all(seen[(idx < 0) & (idx % 2 != 0)] == 0)
    assert np.all(seen[~((idx < 0) & (idx % 2 != 0))] == 1)


def test_drag_coefficients_through_motion():  # test/test_particles.jl:96-97
    """coeff(Linear, Rep) = 1 and coeff(Nonlinear, 1.0) = 1.15: a particle at rest
    at the origin of a uniform unit U (interpolation weights are exact) with
    diam = Re = 1 has Rep = 1, so dudt = coeff * taui."""
    for drag, key in ((_abi.DRAG_LINEAR, "linear_Rep1"), (_abi.DRAG_NONLINEAR, "nonlinear_Rep1")):
        cfg = make_config(16, species=[{"n": 1, "density_ratio": 18.0, "drag": drag, "gravity": 9.8}], Re=1.0)
        with OracleEngine(cfg) as e:
            h = e.haloed_shape
            e.field_set(_abi.FIELD_U, np.ones(h), haloed=True)
            e.field_set(_abi.FIELD_V, np.zeros(h), haloed=True)
            e.field_set(_abi.FIELD_W, np.zeros(h), haloed=True)
            z = np.zeros(1)
            e.upload_particles(0, np.ones(1), z, z, z, z, z, z)
            e.particles_motion(0, 1)
            taup = 1.0 / 18.0 * 18.0 * 1.0 * (1.0 * 1.0)
            expect = KA["drag"][key] * (1.0 - 0.0) * (1.0 / taup) - 9.8
            assert e.prop_get(0, _abi.PROP_DUDT)[0] == expect


def test_periodic_halo_fill_invariant():  # lib/topologies/test/test_mpi.jl:40-53
    n, h = 6, 3
    cfg = make_config(n, mode=_abi.MODE_FLOW)
    with OracleEngine(cfg) as e:
        g = np.arange(1, n ** 3 + 1, dtype=np.float64).reshape(n, n, n)
        A = np.zeros(e.haloed_shape)
        A[h:h + n, h:h + n, h:h + n] = g
        e.field_set(_abi.FIELD_U, A, haloed=True)
        e.synchalo([_abi.FIELD_U], h, True)
        got = e.field_get(_abi.FIELD_U, haloed=True)
        idx = (np.arange(1 - h, n + h + 1) - 1) % n  # mod1 - 1
        assert np.array_equal(got, g[np.ix_(idx, idx, idx)])
        # FaceHalo: only cells with a single out-of-range index are filled
        e.field_set(_abi.FIELD_V, A, haloed=True)
        e.synchalo([_abi.FIELD_V], 1, False)
        got = e.field_get(_abi.FIELD_V, haloed=True)
        assert got[h - 1, h, h] == g[n - 1, 0, 0] and got[h - 1, h - 1, h] == 0.0


def test_particle_periodic_wrap_invariant():  # test/test_particles_mpi.jl:46-61
    n = 64
    cfg = make_config(16, species=[{"n": n}])
    L = 2 * math.pi
    rng = np.random.default_rng(3)
    x = rng.uniform(-L, 2 * L, n)
    y = rng.uniform(-L, 2 * L, n)
    z = rng.uniform(-0.99 * L, 1.99 * L, n)
    with OracleEngine(cfg) as e:
        o = np.zeros(n)
        e.upload_particles(0, np.ones(n), x, y, z, o, o, o)
        partner = rng.random(n)
        e.prop_set(0, _abi.PROP_X2, partner)
        e.particles_boundary(0, 1)
        X = e.prop_get(0, _abi.PROP_X)
        assert np.all((X >= 0) & (X <= L))
        shift = np.where(x < 0, L, np.where(x >= L, -L, 0.0))
        assert np.array_equal(X, x + shift)
        assert np.array_equal(e.prop_get(0, _abi.PROP_X2), partner + shift)


def test_searchsorted_samples():  # test/test_utils.jl:78-94
    """The binary searches of src/utils/fast.jl:8-40 (the oracle's starts and
    stops) on the reference's samples, against Base's definitions
    (searchsortedfirst = bisect_left + 1, searchsortedlast = bisect_right)."""
    import bisect
    import ctypes as C

    lib = load_oracle()
    f = lib.lcs_oracle_searchsorted
    f.restype = None
    f.argtypes = [C.POINTER(C.c_int64), C.c_int64, C.c_int64, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    samples = KA["searchsorted"]["samples"]
    assert len(samples) == 11
    for smp in samples:
        v, x = smp["v"], smp["x"]
        arr = (C.c_int64 * max(1, len(v)))(*v)
        a, b = C.c_int64(), C.c_int64()
        f(arr, len(v), x, C.byref(a), C.byref(b))
        assert (a.value, b.value) == (bisect.bisect_left(v, x) + 1, bisect.bisect_right(v, x)), smp


def test_hasher_known_answers_and_round_trip():  # test/test_utils.jl:103-127
    """sub2ind on ranges (1:3, 1:4) and the encode/decode round trip over
    0:5 x 0:5 x 0:5 (LinearIndices), through the oracle's cell hash."""
    import ctypes as C

    lib = load_oracle()
    enc, dec = lib.lcs_oracle_cell_encode, lib.lcs_oracle_cell_decode
    enc.restype, enc.argtypes = C.c_int64, [C.POINTER(C.c_int64), C.POINTER(C.c_int32)]
    dec.restype, dec.argtypes = None, [C.POINTER(C.c_int64), C.c_int64, C.POINTER(C.c_int32)]
    for k in KA["hasher"]["sub2ind"]:  # axes starting at 1: offsets sub - 1
        (l0, h0), (l1, h1) = k["ranges"]
        ln = (C.c_int64 * 3)(h0 - l0 + 1, h1 - l1 + 1, 1)
        ci = (C.c_int32 * 3)(k["sub"][0] - l0, k["sub"][1] - l1, 0)
        assert enc(ln, ci) == k["ind"], k
    ln = (C.c_int64 * 3)(6, 6, 6)
    lin = np.arange(1, 217).reshape((6, 6, 6), order="F")  # LinearIndices((6, 6, 6))
    out = (C.c_int32 * 3)()
    for i in range(6):
        for j in range(6):
            for kk in range(6):
                h = enc(ln, (C.c_int32 * 3)(i, j, kk))
                assert h == lin[i, j, kk]
                dec(ln, h, out)
                assert tuple(out) == (i, j, kk)
