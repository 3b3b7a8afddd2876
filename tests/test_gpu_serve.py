"""The batching and serving forms over the CUDA library: every member of a
batch and every served request gives, bit for bit, the result of the same run
alone (FP64 and FP32-mixed), while their work overlaps on the GPU."""

import pytest

from lcs_b200 import Engine, _abi
from serve_cases import (check_async_equals_step, check_batch_equals_members_alone, check_group_equals_members_alone,
                         check_server, group_configs)

pytestmark = pytest.mark.gpu


def test_async_steps_equal_step():
    check_async_equals_step(Engine, _abi.load_library())


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_FP32_MIXED])
def test_batch_members_equal_solo_runs(precision):
    check_batch_equals_members_alone(Engine, _abi.load_library(), precision=precision)


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_FP32_MIXED])
def test_server_results_equal_solo_runs(precision):
    check_server(Engine, _abi.load_library(), precision=precision)


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_FP32_MIXED])
def test_group_members_equal_solo_runs(precision):
    check_group_equals_members_alone(Engine, _abi.load_library(), precision=precision)


def test_group_of_more_than_one_launch_of_members():
    """26 members: the sweep kernels take 24 members a launch, so a group
    sweep is two launches."""
    check_group_equals_members_alone(Engine, _abi.load_library(), count=26, nsteps=2, n=16)


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_FP32_MIXED])
def test_batch_of_one_shape_runs_as_groups(precision):
    """Members of one shape share launch shapes, so the batch steps them as a
    group; each equals its solo run with the same launch shapes."""
    check_batch_equals_members_alone(Engine, _abi.load_library(), precision=precision,
                                     cfgs=group_configs(precision, count=6))


def test_group_rejects_mixed_shapes():
    import ctypes as C

    lib = _abi.load_library()
    from helpers import make_config

    a, b = Engine(make_config(16)), Engine(make_config(24))
    hs = (C.c_void_p * 2)(a.handle.value, b.handle.value)
    grp = C.c_void_p()
    assert lib.lcs_group_create(hs, 2, C.byref(grp)) == _abi.EINVAL
    a.close()
    b.close()
