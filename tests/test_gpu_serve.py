"""The batching and serving forms over the CUDA library: every member of a
batch and every served request gives, bit for bit, the result of the same run
alone (FP64 and FP32-mixed), while their work overlaps on the GPU."""

import pytest

from lcs_b200 import Engine, _abi
from serve_cases import check_async_equals_step, check_batch_equals_members_alone, check_server

pytestmark = pytest.mark.gpu


def test_async_steps_equal_step():
    check_async_equals_step(Engine, _abi.load_library())


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_FP32_MIXED])
def test_batch_members_equal_solo_runs(precision):
    check_batch_equals_members_alone(Engine, _abi.load_library(), precision=precision)


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_FP32_MIXED])
def test_server_results_equal_solo_runs(precision):
    check_server(Engine, _abi.load_library(), precision=precision)
