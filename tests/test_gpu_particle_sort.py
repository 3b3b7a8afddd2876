"""The particle sort (lcs_set_particle_sort) on the CUDA library: each particle
equals the unsorted run bit for bit, and the sorted order and values equal the
oracle's (FP64, no forcing: both libraries agree to the last bit)."""

import numpy as np
import pytest

from lcs_b200 import Engine, _abi
from oracle_engine import OracleEngine
from sort_cases import check_group_sort_equals_alone, check_sort_keeps_values, run, sort_config

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("graphs", [0, 1])
def test_sort_keeps_every_particle(graphs):
    check_sort_keeps_values(Engine, nsteps=4, interval=2, graphs=graphs)


def test_sort_in_asynchronous_steps():
    check_sort_keeps_values(Engine, nsteps=3, interval=3, graphs=1, use_async=True)


def test_sort_fp32_mixed():
    check_sort_keeps_values(Engine, nsteps=4, interval=2, graphs=1, precision=_abi.PRECISION_FP32_MIXED)


@pytest.mark.parametrize("interval", [1, 3])
def test_sorted_run_equals_oracle(interval):
    cfg = sort_config(graphs=1)
    d = run(Engine, cfg, 11, 5, interval)
    o = run(OracleEngine, sort_config(graphs=1), 11, 5, interval)
    for fd, fo in zip(d["flow"], o["flow"]):
        assert np.array_equal(fd, fo)
    for s, (pd, po) in enumerate(zip(d["parts"], o["parts"])):
        for k in pd:  # the same order, the same bits
            assert np.array_equal(pd[k], po[k]), (s, k)


def test_group_sorts_its_members():
    check_group_sort_equals_alone(Engine, Engine._load())
