"""Flow and particle statistics on the host, for stating the precision form's
error per statistic (and for users who download a state).

`flow_stat` restates `Flows.stat` (src/flows/stat.jl:66-153) on interior
arrays indexed [k, j, i] (x fastest), periodic: the halo reads of the
reference become periodic shifts.  The derivative stencils are those of
src/diff.jl (diff1_o4_at_half = (a - 27b + 27c - d)/24); the strain-rate
components and means follow stat.jl:83-138 line by line.  `energy_spectrum`
is the shell-summed kinetic energy spectrum of the three components (their
staggering only shifts phases, so |u_hat|^2 is that of the stored values).
"""

from __future__ import annotations

import math

import numpy as np


def _sh(a: np.ndarray, di: int = 0, dj: int = 0, dk: int = 0) -> np.ndarray:
    """a[i+di, j+dj, k+dk] for every (i, j, k), periodic (a is [k, j, i])."""
    return np.roll(a, (-dk, -dj, -di), axis=(0, 1, 2))


def _d1o4(a, b, c, d):
    return (1.0 / 24.0) * (a - 27.0 * b + 27.0 * c - d)


def flow_stat(U: np.ndarray, V: np.ndarray, W: np.ndarray, nu: float, L: float = 2.0 * math.pi) -> dict:
    """`Flows.stat` without the integral length: means, urms, k, epsilon,
    tau_eta, lambda (l_mu), l_eta, Re_lambda, k_eta, skewness, flatness."""
    nz, ny, nx = U.shape
    dxi, dyi, dzi = nx / L, ny / L, nz / L
    dudx = dxi * _d1o4(_sh(U, -2), _sh(U, -1), U, _sh(U, 1))
    dvdy = dyi * _d1o4(_sh(V, 0, -2), _sh(V, 0, -1), V, _sh(V, 0, 1))
    dwdz = dzi * _d1o4(_sh(W, 0, 0, -2), _sh(W, 0, 0, -1), W, _sh(W, 0, 0, 1))
    dudy = dyi * _d1o4(_sh(U, 0, -2), _sh(U, 0, -1), U, _sh(U, 0, 1))
    dvdx = dxi * _d1o4(_sh(V, -1, -1), _sh(V, 0, -1), _sh(V, 1, -1), _sh(V, 2, -1))
    dvdz = dzi * _d1o4(_sh(V, 0, -1, -1), _sh(V, 0, -1, 0), _sh(V, 0, -1, 1), _sh(V, 0, -1, 2))
    dwdy = dyi * _d1o4(_sh(W, 0, -2), _sh(W, 0, -1), W, _sh(W, 0, 1))
    dwdx = dxi * _d1o4(_sh(W, -1, 0, -1), _sh(W, 0, 0, -1), _sh(W, 1, 0, -1), _sh(W, 2, 0, -1))
    dudz = dzi * _d1o4(_sh(U, 0, 0, -2), _sh(U, 0, 0, -1), U, _sh(U, 0, 0, 1))
    s11, s22, s33 = dudx, dvdy, dwdz  # 0.5 * (a + a)
    s12 = 0.5 * (dudy + dvdx)
    s13 = 0.5 * (dudz + dwdx)
    s23 = 0.5 * (dvdz + dwdy)
    s2 = (2.0 * (s11 ** 2 + s22 ** 2 + s33 ** 2 + 2.0 * (s12 ** 2 + s13 ** 2 + s23 ** 2))).mean()
    u2 = (U ** 2 + V ** 2 + W ** 2).mean()
    d2, d3, d4 = (dudx ** 2).mean(), (dudx ** 3).mean(), (dudx ** 4).mean()
    um, vm, wm = U.mean(), V.mean(), W.mean()
    urms = math.sqrt(u2 / 3.0)
    k = 0.5 * (u2 - um ** 2 - vm ** 2 - wm ** 2)
    Re = 1.0 / nu
    eps = s2 / Re
    tau_eta = math.sqrt(1.0 / eps / Re)
    l_mu = math.sqrt(15.0 * urms ** 2 / eps / Re)
    l_eta = (1.0 / eps / Re ** 3) ** 0.25
    re_lambda = l_mu * urms * Re
    n = min(nx, ny, nz)
    return {"u_mean": um, "v_mean": vm, "w_mean": wm, "urms": urms, "k": k, "epsilon": eps, "tau_eta": tau_eta,
            "l_mu": l_mu, "l_eta": l_eta, "Re_lambda": re_lambda, "k_eta": (n / 2.0) * l_eta,
            "skewness": -d3 / d2 ** 1.5, "flatness": d4 / d2 ** 2}


def energy_spectrum(U: np.ndarray, V: np.ndarray, W: np.ndarray) -> np.ndarray:
    """E(k) for integer shells k = 0 .. n/2: sum of 0.5 |u_hat|^2 over wave
    vectors with round(|k|) = k (u_hat = FFT(u) / n^3)."""
    nz, ny, nx = U.shape
    kz = np.fft.fftfreq(nz, 1.0 / nz)
    ky = np.fft.fftfreq(ny, 1.0 / ny)
    kx = np.fft.rfftfreq(nx, 1.0 / nx)
    kk = np.sqrt(kz[:, None, None] ** 2 + ky[None, :, None] ** 2 + kx[None, None, :] ** 2)
    shell = np.rint(kk).astype(np.int64)
    # rfft stores half of x: the modes with 0 < kx < nx/2 stand for two
    weight = np.full(kx.shape, 2.0)
    weight[0] = 1.0
    if nx % 2 == 0:
        weight[-1] = 1.0
    nbins = int(shell.max()) + 1
    e = np.zeros(nbins)
    norm = float(nx * ny * nz)
    try:
        import os

        import scipy.fft as sfft

        def rfftn(a):
            return sfft.rfftn(a, workers=os.cpu_count() or 1)
    except ImportError:
        rfftn = np.fft.rfftn
    for a in (U, V, W):
        h = rfftn(a) / norm
        e3 = 0.5 * (h.real ** 2 + h.imag ** 2) * weight[None, None, :]
        e += np.bincount(shell.ravel(), weights=e3.ravel(), minlength=nbins)
    kmax = min(nx, ny, nz) // 2
    return e[: kmax + 1]


def particle_rms_velocity(u: np.ndarray, v: np.ndarray, w: np.ndarray) -> float:
    """sqrt(<u^2 + v^2 + w^2> / 3), the particles' urms."""
    return math.sqrt(float(np.mean(u * u + v * v + w * w)) / 3.0)
