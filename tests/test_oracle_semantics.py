"""Independent restatements (plain Python/numpy, written from the reference's
Julia source) that check the C oracle at tiny sizes.  Element-wise stages are
compared bit for bit; reductions to 1e-14."""

import math

import numpy as np
import pytest

from helpers import load_particles, load_random_flow, make_config, rel_l2
from lcs_b200 import _abi
from oracle_engine import OracleEngine

F = _abi


class Grid:
    """Haloed numpy arrays [k, j, i]; logical index i -> i + h - 1."""

    def __init__(self, n, h):
        self.n, self.h = n, h

    def ix(self, i):
        return i + self.h - 1


def o4(a, b, c, d):
    return (1 / 16) * (-a + 9 * b + 9 * c - d)


def o2(a, b):
    return (1 / 2) * (a + b)


def d2o4(a, b, c, d, e):
    return (1 / 12) * (-a + 16 * b - 30 * c + 16 * d - e)


def sflux(j1a, j1b, j3a, j3b):
    return (9 / 8) * (-j1a + j1b) - (1 / 8) * (1 / 3) * (-j3a + j3b)


def rhs_numpy(U, V, W, P, n, h, Re):
    """Flows.rhs! (src/flows/rhs.jl:44-252) with numpy slices."""
    dx = 2 * math.pi / n
    dxi = 1 / dx
    Rei = 1 / Re
    S = U.shape[0]

    def sl(a, off, axis, lo, hi):
        # values A[logical lo+off .. hi+off] along axis, logical lo..hi on the others
        idx = [slice(lo + h - 1, hi + h) for _ in range(3)]
        ax = 2 - axis  # numpy axis of logical axis (x=2, y=1, z=0)
        idx[ax] = slice(lo + h - 1 + off, hi + h + off)
        return a[tuple(idx)]

    out = []
    vel = (U, V, W)
    for comp in range(3):
        A = vel[comp]
        lo1, hi1 = -1, n + 1
        uc = o4(*(sl(vel[0], o, comp, lo1, hi1) for o in (-1, 0, 1, 2)))
        vc = o4(*(sl(vel[1], o, comp, lo1, hi1) for o in (-1, 0, 1, 2)))
        wc = o4(*(sl(vel[2], o, comp, lo1, hi1) for o in (-1, 0, 1, 2)))
        a1 = [o2(sl(A, 0, ax, lo1, hi1), sl(A, 1, ax, lo1, hi1)) for ax in range(3)]
        a3 = [o2(sl(A, -1, ax, lo1, hi1), sl(A, 2, ax, lo1, hi1)) for ax in range(3)]
        J1 = [uc * a1[0], vc * a1[1], wc * a1[2]]
        J3 = [uc * a3[0], vc * a3[1], wc * a3[2]]
        diff = (dxi ** 2 * d2o4(*(sl(A, o, 0, 1, n) for o in (-2, -1, 0, 1, 2)))
                + dxi ** 2 * d2o4(*(sl(A, o, 1, 1, n) for o in (-2, -1, 0, 1, 2)))
                + dxi ** 2 * d2o4(*(sl(A, o, 2, 1, n) for o in (-2, -1, 0, 1, 2)))) * Rei
        pres = dxi * (-sl(P, 0, comp, 1, n) + sl(P, 1, comp, 1, n))
        d = diff - pres
        # J arrays are stored on -1..n+1; read them at offsets relative to 1..n
        def js(Jarr, off, axis):
            idx = [slice(2, 2 + n) for _ in range(3)]  # logical 1..n within -1..n+1 starts at index 2
            ax = 2 - axis
            idx[ax] = slice(2 + off, 2 + off + n)
            return Jarr[tuple(idx)]
        adv = (dxi * sflux(js(J1[0], -1, 0), js(J1[0], 0, 0), js(J3[0], -2, 0), js(J3[0], 1, 0))
               + dxi * sflux(js(J1[1], -1, 1), js(J1[1], 0, 1), js(J3[1], -2, 1), js(J3[1], 1, 1))
               + dxi * sflux(js(J1[2], -1, 2), js(J1[2], 0, 2), js(J3[2], -2, 2), js(J3[2], 1, 2)))
        out.append(d - adv)
    return out


@pytest.mark.parametrize("stage", [1, 2])
def test_rhs_matches_numpy_restatement(stage):
    n, Re = 8, 1.0
    cfg = make_config(n, mode=F.MODE_FLOW)
    with OracleEngine(cfg) as e:
        rng = np.random.default_rng(11)
        fields = {}
        for f in (F.FIELD_U, F.FIELD_V, F.FIELD_W, F.FIELD_U2, F.FIELD_V2, F.FIELD_W2, F.FIELD_P):
            fields[f] = rng.random(e.haloed_shape)
            e.field_set(f, fields[f], haloed=True)
        e.rhs(stage)
        base = 0 if stage == 1 else 3
        ref = rhs_numpy(fields[base], fields[base + 1], fields[base + 2], fields[F.FIELD_P], n, 3, Re)
        for c in range(3):
            assert np.array_equal(e.field_get(F.FIELD_DUDT + c), ref[c])


def synchalo_py(A, n, h, r, full=True):
    N = A.shape[0]
    for k in range(1 - r, n + r + 1):
        for j in range(1 - r, n + r + 1):
            for i in range(1 - r, n + r + 1):
                out = [(x < 1 or x > n) for x in (i, j, k)]
                if not any(out) or (not full and sum(out) != 1):
                    continue
                w = [(x - 1) % n + 1 for x in (i, j, k)]
                A[k + h - 1, j + h - 1, i + h - 1] = A[w[2] + h - 1, w[1] + h - 1, w[0] + h - 1]
    assert N == n + 2 * h


def hsmac_py(U, V, W, P, n, h, cfg, dt):
    """Flows.couple!(::HSMAC) (src/flows/couples/hsmac.jl) with plain loops."""
    dx = 2 * math.pi / n
    dxi = dyi = dzi = 1 / dx
    dl = 1 / (2 * (dxi ** 2 + dyi ** 2 + dzi ** 2))
    omega = cfg.omega
    dti = 1 / dt
    dxmin = dx
    Div2 = np.zeros_like(U)
    X = lambda a: a + h - 1

    def cell(i, j, k):
        dudx = dxi * (-U[X(k), X(j), X(i - 1)] + U[X(k), X(j), X(i)])
        dvdy = dyi * (-V[X(k), X(j - 1), X(i)] + V[X(k), X(j), X(i)])
        dwdz = dzi * (-W[X(k - 1), X(j), X(i)] + W[X(k), X(j), X(i)])
        div = dudx + dvdy + dwdz
        dp = -omega * div * dl
        Div2[X(k), X(j), X(i)] = div ** 2
        P[X(k), X(j), X(i)] += dp * dti
        U[X(k), X(j), X(i - 1)] -= dp * dxi
        U[X(k), X(j), X(i)] += dp * dxi
        V[X(k), X(j - 1), X(i)] -= dp * dyi
        V[X(k), X(j), X(i)] += dp * dyi
        W[X(k - 1), X(j), X(i)] -= dp * dzi
        W[X(k), X(j), X(i)] += dp * dzi

    def foraxes(box):
        (x0, x1), (y0, y1), (z0, z1) = box
        for color in (0, 1):
            for k in range(z0, z1 + 1):
                for j in range(y0, y1 + 1):
                    for i in range(x0, x1 + 1):
                        if (i + j + k) % 2 == color:  # RedBlackFast selects true parity
                            cell(i, j, k)

    def faces(d, c):
        (dx0, dx1), (dy0, dy1), (dz0, dz1) = d
        (cx0, cx1), (cy0, cy1), (cz0, cz1) = c
        return [((dx0, dx1), (dy0, dy1), (dz0, cz0 - 1)), ((dx0, dx1), (dy0, dy1), (cz1 + 1, dz1)),
                ((dx0, dx1), (dy0, cy0 - 1), (cz0, cz1)), ((dx0, dx1), (cy1 + 1, dy1), (cz0, cz1)),
                ((dx0, cx0 - 1), (cy0, cy1), (cz0, cz1)), ((cx1 + 1, dx1), (cy0, cy1), (cz0, cz1))]

    def resid():
        s = None
        for k in range(1, n + 2):
            for j in range(1, n + 2):
                for i in range(1, n + 2):
                    v = Div2[X(k), X(j), X(i)]
                    s = v if s is None else s + v
        return math.sqrt(s / (n + 1) ** 3)

    box = lambda a, b: ((a, n + b),) * 3
    itr, div = 0, 0.0
    if cfg.time_blocking:
        d1, d2, d3, core = box(-1, 3), box(0, 2), box(1, 1), box(2, 0)
        while itr < cfg.itrmax:
            if not cfg.overlap:
                for A in (U, V, W):
                    synchalo_py(A, n, h, h)
            for d in (d1, d2, d3):
                if cfg.overlap and d is d1:
                    for A in (U, V, W):
                        synchalo_py(A, n, h, h)
                    foraxes(core)
                    for f in faces(d1, core):
                        foraxes(f)
                else:
                    foraxes(d)
                div = resid()
                if div * dxmin < cfg.epsp and cfg.itrmin <= itr:
                    return itr, div
                itr += 1
    else:
        d, core = box(1, 1), box(2, 0)
        while itr < cfg.itrmax:
            if cfg.overlap:
                for A in (U, V, W):
                    synchalo_py(A, n, h, 1)
                foraxes(core)
                for f in faces(d, core):
                    foraxes(f)
            else:
                for A in (U, V, W, P):
                    synchalo_py(A, n, h, 1)
                foraxes(d)
            div = resid()
            if div * dxmin < cfg.epsp and cfg.itrmin <= itr:
                break
            itr += 1
    return itr, div


@pytest.mark.parametrize("time_blocking", [True, False])
@pytest.mark.parametrize("overlap", [True, False])
def test_hsmac_matches_loop_restatement(time_blocking, overlap):
    n, h = 4, 3
    cfg = make_config(n, mode=F.MODE_FLOW, time_blocking=time_blocking, overlap=overlap, itrmin=2, itrmax=6,
                      epsp=1e-3)
    dt = 0.01
    with OracleEngine(cfg) as e:
        rng = np.random.default_rng(5)
        U, V, W, P = (rng.random(e.haloed_shape) for _ in range(4))
        for f, a in zip((F.FIELD_U, F.FIELD_V, F.FIELD_W, F.FIELD_P), (U, V, W, P)):
            e.field_set(f, a, haloed=True)
        log = e.couple(2, dt)
        itr, div = hsmac_py(U, V, W, P, n, h, cfg, dt)
        assert log["itr"] == itr
        assert abs(log["div"] - div) <= 1e-14 * div
        for f, a in zip((F.FIELD_U, F.FIELD_V, F.FIELD_W, F.FIELD_P), (U, V, W, P)):
            assert np.array_equal(e.field_get(f), a[h:h + n, h:h + n, h:h + n])


def interp_py(A, h, i, j, k, r1, r2, r3):
    X = lambda a: a + h - 1
    c = lambda di, dj, dk: A[X(k + dk), X(j + dj), X(i + di)]
    return ((1 - r1) * (1 - r2) * (1 - r3) * c(0, 0, 0) + r1 * (1 - r2) * (1 - r3) * c(1, 0, 0)
            + r1 * r2 * (1 - r3) * c(1, 1, 0) + (1 - r1) * r2 * (1 - r3) * c(0, 1, 0)
            + (1 - r1) * (1 - r2) * r3 * c(0, 0, 1) + r1 * (1 - r2) * r3 * c(1, 0, 1)
            + r1 * r2 * r3 * c(1, 1, 1) + (1 - r1) * r2 * r3 * c(0, 1, 1))


def test_particle_motion_and_update_match_restatement():
    n, npart = 16, 50
    cfg = make_config(n, species=[{"n": npart, "density_ratio": 2.5, "gravity": 9.8, "drag": F.DRAG_NONLINEAR}],
                      Re=3.0)
    with OracleEngine(cfg) as e:
        fl = load_random_flow([e], seed=2, fields=(F.FIELD_U, F.FIELD_V, F.FIELD_W))
        load_particles([e], 0, npart, seed=4, diam=0.3)
        x, y, z = (e.prop_get(0, p) for p in (F.PROP_X, F.PROP_Y, F.PROP_Z))
        u, v, w = (e.prop_get(0, p) for p in (F.PROP_U, F.PROP_V, F.PROP_W))
        e.particles_motion(0, 1)
        du = e.prop_get(0, F.PROP_DUDT)
        dx = 2 * math.pi / n
        Re = 3.0
        for p in range(npart):
            xi, yi, zi = x[p], y[p], z[p]
            uf = interp_py(fl[0], 3, math.floor(xi / dx), math.floor(yi / dx + 0.5), math.floor(zi / dx + 0.5),
                           xi / dx - math.floor(xi / dx), yi / dx - math.floor(yi / dx + 0.5) + 0.5,
                           zi / dx - math.floor(zi / dx + 0.5) + 0.5)
            vf = interp_py(fl[1], 3, math.floor(xi / dx + 0.5), math.floor(yi / dx), math.floor(zi / dx + 0.5),
                           xi / dx - math.floor(xi / dx + 0.5) + 0.5, yi / dx - math.floor(yi / dx),
                           zi / dx - math.floor(zi / dx + 0.5) + 0.5)
            wf = interp_py(fl[2], 3, math.floor(xi / dx + 0.5), math.floor(yi / dx + 0.5), math.floor(zi / dx),
                           xi / dx - math.floor(xi / dx + 0.5) + 0.5, yi / dx - math.floor(yi / dx + 0.5) + 0.5,
                           zi / dx - math.floor(zi / dx))
            vrel = math.sqrt((uf - u[p]) ** 2 + (vf - v[p]) ** 2 + (wf - w[p]) ** 2)
            Rep = 0.3 * vrel * Re
            f = 1.0 + 0.15 * Rep ** 0.687
            taup = 1 / 18 * 2.5 * Re * 0.3 ** 2
            assert du[p] == f * (uf - u[p]) * (1 / taup) - 9.8
        # update stage 1: x2 = x + dt u, u2 = u + dt dudt (src/particles/update.jl)
        e.particles_update(0, 1, 0.005)
        assert np.array_equal(e.prop_get(0, F.PROP_X2), x + 0.005 * u)
        assert np.array_equal(e.prop_get(0, F.PROP_U2), u + 0.005 * du)


def test_timestep_matches_numpy():
    n = 8
    cfg = make_config(n, mode=F.MODE_FLOW, Re=50.0, cfl=0.3, dtmax=1.0)
    with OracleEngine(cfg) as e:
        rng = np.random.default_rng(9)
        U, V, W = (rng.standard_normal(e.interior_shape) for _ in range(3))
        for f, a in zip((F.FIELD_U, F.FIELD_V, F.FIELD_W), (U, V, W)):
            e.field_set(f, a)
        dt = e.flow_timestep()
        Uw = lambda a, s, ax: np.roll(a, s, axis=ax)
        uc = o4(Uw(U, 2, 2), Uw(U, 1, 2), U, Uw(U, -1, 2))
        vc = o4(Uw(V, 2, 1), Uw(V, 1, 1), V, Uw(V, -1, 1))
        wc = o4(Uw(W, 2, 0), Uw(W, 1, 0), W, Uw(W, -1, 0))
        dx = 2 * math.pi / n
        c = [1.0, 0.3 * dx / (np.abs(uc).max() + 1e-10), 0.3 * dx / (np.abs(vc).max() + 1e-10),
             0.3 * dx / (np.abs(wc).max() + 1e-10), 0.5 * (dx / 2) ** 2 / (1 / 50.0)]
        assert dt == min(c)


def test_linear_forcing_matches_numpy():
    n = 8
    cfg = make_config(n, mode=F.MODE_FLOW, forcing=F.FORCING_LINEAR_POWER, power=0.5)
    with OracleEngine(cfg) as e:
        rng = np.random.default_rng(12)
        U, V, W = (rng.random(e.interior_shape) for _ in range(3))
        for f, a in zip((F.FIELD_U, F.FIELD_V, F.FIELD_W), (U, V, W)):
            e.field_set(f, a)
        dt = 0.01
        out = e.forcing(dt)
        uu = o2(np.roll(U, 1, 2), U)
        vv = o2(np.roll(V, 1, 1), V)
        ww = o2(np.roll(W, 1, 0), W)
        u2 = (uu * uu + vv * vv + ww * ww).mean()
        um, vm, wm = U.mean(), V.mean(), W.mean()
        A = 0.5 / (2 * (0.5 * (u2 - um ** 2 - vm ** 2 - wm ** 2)))
        us, vs, ws = A * (U - um), A * (V - vm), A * (W - wm)
        p = (U * us + V * vs + W * ws).mean()
        assert abs(out["p"] - p) < 1e-13 * abs(p)
        assert rel_l2(e.field_get(F.FIELD_U), U + us * dt) < 1e-14


def test_rcf_forcing_matches_numpy_fft():
    n, cs, kmin, kmax, e10 = 16, 4, 1, 2, 1.0
    cfg = make_config(n, mode=F.MODE_FLOW, forcing=F.FORCING_RC_ENERGY, energy=e10, kmin=kmin, kmax=kmax, coarse=cs)
    from oracle_engine import load_oracle
    lib = load_oracle()
    with OracleEngine(cfg) as e:
        rng = np.random.default_rng(13)
        Us = [rng.random(e.interior_shape) for _ in range(3)]
        for f, a in enumerate(Us):
            e.field_set(f, a)
        dt = 0.02
        out = e.forcing(dt)
        f = n // cs
        phi = f / 2
        src = []
        for a in Us:
            coarse = a.reshape(cs, f, cs, f, cs, f).mean(axis=(1, 3, 5))
            hat = np.fft.rfftn(coarse)  # [kz, ky, kx]
            for k0 in range(kmin, kmax + 1):
                pass
            src.append(hat)
        # shell rescale with energies summed over all three components
        def coef(hat, kx, ky, kz):
            return hat[kz % cs, ky % cs, kx] / cs ** 3
        r = {}
        for k0 in range(kmin, kmax + 1):
            en = 0.0
            for kz in range(-k0, k0 + 1):
                for ky in range(-k0, k0 + 1):
                    for kx in range(0, k0 + 1):
                        if (k0 - .5) ** 2 <= kx * kx + ky * ky + kz * kz < (k0 + .5) ** 2:
                            w = 1 if kx == 0 else 2
                            en += w * sum(abs(coef(h, kx, ky, kz)) ** 2 for h in src)
            en /= 2
            r[k0] = math.sqrt(lib.lcs_oracle_enespe0(k0, e10) / max(en, 1e-8)) - 1
        x = np.arange(1, n + 1)
        ph = np.exp(1j * np.pi * 2 * (x - phi) / n)
        fields = []
        for a, h in zip(Us, src):
            s = np.zeros((n, n, n))
            for kz in range(-kmax, kmax + 1):
                for ky in range(-kmax, kmax + 1):
                    for kx in range(0, kmax + 1):
                        k2 = kx * kx + ky * ky + kz * kz
                        shell = [k0 for k0 in r if (k0 - .5) ** 2 <= k2 < (k0 + .5) ** 2]
                        if not shell:
                            continue
                        c = coef(h, kx, ky, kz) * r[shell[0]]
                        canon = next((v for v in (kx, ky, kz) if v != 0), 0) > 0
                        if not canon:
                            continue
                        e3 = (ph[None, None, :] ** kx) * (ph[None, :, None] ** ky) * (ph[:, None, None] ** kz)
                        s += 2 * (c * e3).real
            fields.append(s)
        p = ((Us[0] * fields[0] + Us[1] * fields[1] + Us[2] * fields[2]) / dt).mean()
        assert abs(out["p"] - p) < 1e-11 * abs(p)
        assert out["e10"] == e10
        for c in range(3):
            assert rel_l2(e.field_get(c), Us[c] + fields[c]) < 1e-13


def test_oracle_evolve_two_steps():
    n = 16
    cfg = make_config(n, forcing=F.FORCING_LINEAR_POWER, power=0.5, Re=100.0, itrmax=30, epsp=1e-6,
                      species=[{"n": 100, "density_ratio": 843.0}])
    from lcs_b200 import inits
    with OracleEngine(cfg) as e:
        U, V, W, P = inits.spectral_flow(n, seed=1)
        e.upload_flow(U, V, W, P)
        x, y, z = inits.random_positions(100, 3)
        o = np.zeros(100)
        e.upload_particles(0, np.full(100, 0.05), x, y, z, o, o, o)
        e.init_particle_velocity(0)
        logs = e.step(2)
        assert [lg["step"] for lg in logs] == [1, 2]
        for lg in logs:
            assert lg["dt"] > 0 and math.isfinite(lg["forcing"]["p"])
            assert lg["couple1"]["itr"] >= 6 and lg["couple2"]["itr"] >= 6
        Ud = e.download_flow()[0]
        assert np.all(np.isfinite(Ud))
