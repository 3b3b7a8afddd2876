"""Host-side initial conditions (src/flows/inits, src/particles/init.jl).

`ideal_flow` restates the reference's analytic init.  `spectral_flow` and
the random particle positions are new seeded generators (numpy PCG64); the
reference's `random-flow` uses Julia's Xoshiro stream, which cannot be
reproduced here.
"""

from __future__ import annotations

import math

import numpy as np

TWO_PI = 2.0 * math.pi


def ideal_flow(n: int):
    """`init!(::IdealFlow)` (src/flows/inits/idealflow.jl:5-49); arrays [k, j, i]."""
    dx = TWO_PI / n
    idx = np.arange(1, n + 1, dtype=np.float64)
    x = dx * (idx - 0.5)
    xg = x[None, None, :]
    yg = x[None, :, None]
    zg = x[:, None, None]
    al, bl = 1.0, 1.0
    Al, Bl = math.sqrt(1.5) * 2.0, -math.sqrt(1.5) * 2.0
    as_, bs, cs = 1.0 * (n / 2), 1.0 * (n / 2), 1.0 * (n / 2)
    As, Cs = math.sqrt(1.5e-2) * 2.0, -math.sqrt(1.5e-2) * 2.0
    ul = Al * np.cos(al * (xg + 0.5 * dx)) * np.sin(bl * yg)
    vl = Bl * np.sin(al * xg) * np.cos(bl * (yg + 0.5 * dx))
    us = As * np.cos(as_ * (xg + 0.5 * dx)) * np.sin(bs * yg) * np.sin(cs * zg)
    vs = 0.0 * np.sin(as_ * xg) * np.cos(bs * (yg + 0.5 * dx)) * np.sin(cs * zg)
    ws = Cs * np.sin(as_ * xg) * np.sin(bs * yg) * np.cos(cs * (zg + 0.5 * dx))
    shape = (n, n, n)
    U = np.broadcast_to(ul + us, shape).copy()
    V = np.broadcast_to(vl + vs, shape).copy()
    W = np.broadcast_to(0.0 * xg + ws, shape).copy()
    return U, V, W, np.zeros(shape)


def spectral_flow(n: int, seed: int = 0, urms: float = 1.0, kpeak: float = 4.0, dtype=np.complex128):
    """Seeded random-phase solenoidal field with E(k) ~ k^4 exp(-2 (k/kpeak)^2).

    A complex Gaussian vector field is projected onto the plane normal to k,
    given amplitude |u_k| ~ k exp(-(k/kpeak)^2) (shell energy 4 pi k^2 |u_k|^2
    ~ E(k)), and evaluated at the staggered points of each component --
    U at (i dx, (j-1/2) dy, (k-1/2) dz), V at ((i-1/2) dx, j dy, (k-1/2) dz),
    W at ((i-1/2) dx, (j-1/2) dy, k dz) (src/particles/interp.jl:92-126) --
    by a phase shift (a product of per-axis phases) before the inverse FFT.
    The real part is kept and the three components are scaled together so
    that sqrt(<U^2+V^2+W^2>/3) = urms.  Returns U, V, W, P (P = 0) indexed
    [k, j, i].  The inverse FFTs use every host core when SciPy is present.
    """
    import os

    try:
        import scipy.fft as sfft

        def ifftn(a):
            return sfft.ifftn(a, workers=os.cpu_count() or 1, overwrite_x=True)
    except ImportError:  # numpy's FFT (one thread)
        ifftn = np.fft.ifftn
    rng = np.random.default_rng(seed)
    k1 = np.fft.fftfreq(n, d=1.0 / n)
    kz = k1[:, None, None]
    ky = k1[None, :, None]
    kx = k1[None, None, :]
    kk2 = kx * kx + ky * ky + kz * kz
    amp = np.sqrt(kk2) * np.exp(-kk2 / (kpeak * kpeak))
    amp[0, 0, 0] = 0.0
    a = []
    for _ in range(3):
        c = rng.standard_normal((n, n, n)).astype(np.complex128)
        c.imag = rng.standard_normal((n, n, n))
        a.append(c)
    kk2[0, 0, 0] = 1.0
    dot = kx * a[0]
    dot += ky * a[1]
    dot += kz * a[2]
    dot /= kk2
    del kk2
    dx = TWO_PI / n
    # phase shifts taking grid point m*dx to the staggered positions
    shifts = [(dx, 0.5 * dx, 0.5 * dx), (0.5 * dx, dx, 0.5 * dx), (0.5 * dx, 0.5 * dx, dx)]
    ks = (kx, ky, kz)
    out = []
    for c in range(3):
        sx, sy, sz = shifts[c]
        comp = a[c]
        comp -= ks[c] * dot
        comp *= amp
        comp *= np.exp(1j * kx * sx)
        comp *= np.exp(1j * ky * sy)
        comp *= np.exp(1j * kz * sz)
        a[c] = None
        f = ifftn(comp.astype(dtype, copy=False)).real * float(n ** 3)
        del comp
        out.append(np.ascontiguousarray(f, dtype=np.float64))
    del dot, a
    e = float(np.mean(out[0] * out[0] + out[1] * out[1] + out[2] * out[2])) / 3.0
    scale = urms / math.sqrt(e)
    for f in out:
        f *= scale
    U, V, W = out
    return U, V, W, np.zeros((n, n, n))


def random_positions(nvalid: int, seed: int):
    """`init_position!(::RandomPosition)` (src/particles/init.jl:84-106): uniform
    in [0, 2pi)^3 (x = origin + rand * length), numpy PCG64 instead of Julia's RNG."""
    rng = np.random.default_rng(seed)
    x = rng.random(nvalid) * TWO_PI
    y = rng.random(nvalid) * TWO_PI
    z = rng.random(nvalid) * TWO_PI
    return x, y, z


def generate_ids(nvalid: int, offset: int = 0):
    """`init_id!(::GenerateId)`: 1-based ids offset by the preceding ranks' counts."""
    return np.arange(1 + offset, nvalid + 1 + offset, dtype=np.int64)
