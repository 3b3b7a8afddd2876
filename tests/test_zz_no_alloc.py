"""The allocation-free time-step entry point (lcs_flow_timestep_noalloc).

It exists for callers that cannot let a library allocate device memory: a
program recording a CUDA stream capture, or one whose device memory belongs to
another allocator.  They hand it U, V, W device arrays they own, in the
reference's haloed layout, and a device double for the result.  Here torch
owns those buffers.  The result must equal the handle-based lcs_flow_timestep
on the same fields, bit for bit (the time step is a max and a min), on two
calls in a row, since every call shares the library's static scratch.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""

import ctypes as C

import numpy as np
import pytest

from helpers import make_config
from lcs_b200 import Engine, _abi

pytestmark = pytest.mark.gpu


def haloed(interior, h, fill):
    """The reference's (n+2h)^3 layout around an interior array [k, j, i]."""
    nz, ny, nx = interior.shape
    a = np.full((nz + 2 * h, ny + 2 * h, nx + 2 * h), fill)
    a[h:h + nz, h:h + ny, h:h + nx] = interior
    return a


def test_noalloc_timestep_equals_handle_timestep_twice():
    torch = pytest.importorskip("torch")
    lib = _abi.load_library()
    dims, h, Re, cfl, dtmax = (32, 24, 40), 3, 150.0, 0.3, 1.0
    cdims = (C.c_int32 * 3)(*dims)
    rng = np.random.default_rng(2024)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    results = []
    for call in range(2):
        shape = (dims[2], dims[1], dims[0])
        U, V, W = (rng.standard_normal(shape) * (1.0 + call) for _ in range(3))
        eng = Engine(make_config(dims=dims, mode=_abi.MODE_FLOW, Re=Re, cfl=cfl, dtmax=dtmax))
        for f, a in zip((_abi.FIELD_U, _abi.FIELD_V, _abi.FIELD_W), (U, V, W)):
            eng.field_set(f, a)
        expect = eng.flow_timestep()
        eng.close()
        # halo cells hold huge values: the entry point must read only the interior
        dev = [torch.from_numpy(haloed(a, h, 1e30)).to("cuda") for a in (U, V, W)]
        out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = lib.lcs_flow_timestep_noalloc(*(C.c_void_p(t.data_ptr()) for t in dev), cdims, h, cfl, dtmax, Re,
                                           C.c_void_p(out.data_ptr()), stream)
        assert rc == 0, lib.lcs_last_error(None)
        torch.cuda.synchronize()
        got = float(out.item())
        assert got == expect, (call, got, expect)
        results.append(got)
    assert results[0] != results[1]  # the second call really recomputed


def test_noalloc_rejects_grids_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    lib = _abi.load_library()
    h = 0
    dims = (4, 4, _abi.NOALLOC_MAX_PLANES + 2)
    t = torch.zeros(dims[0] * dims[1] * dims[2], dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = lib.lcs_flow_timestep_noalloc(*(C.c_void_p(t.data_ptr()) for _ in range(3)), (C.c_int32 * 3)(*dims), h,
                                       0.3, 1.0, 100.0, C.c_void_p(out.data_ptr()), None)
    assert rc == _abi.EINVAL
    assert b"z-planes" in lib.lcs_last_error(None)


def test_noalloc_nan_cell_gives_nan_dt():
    """Julia's maximum(abs, U) propagates a NaN: so does the entry point, and
    the handle-based time step agrees."""
    torch = pytest.importorskip("torch")
    lib = _abi.load_library()
    dims, h = (16, 16, 16), 3
    rng = np.random.default_rng(7)
    shape = (dims[2], dims[1], dims[0])
    U, V, W = (rng.standard_normal(shape) for _ in range(3))
    W[4, 5, 6] = np.nan
    dev = [torch.from_numpy(haloed(a, h, 0.0)).to("cuda") for a in (U, V, W)]
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = lib.lcs_flow_timestep_noalloc(*(C.c_void_p(t.data_ptr()) for t in dev), (C.c_int32 * 3)(*dims), h, 0.3,
                                       1.0, 100.0, C.c_void_p(out.data_ptr()), None)
    assert rc == 0, lib.lcs_last_error(None)
    torch.cuda.synchronize()
    assert np.isnan(float(out.item()))
