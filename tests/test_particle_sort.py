"""The particle sort (lcs_set_particle_sort) on the oracle: values kept per
particle, cell order after a sort step, argument errors, grouped steps equal to members alone."""

import pytest

from helpers import make_config
from lcs_b200 import _abi
from lcs_b200.engine import LCSError
from oracle_engine import OracleEngine, load_oracle
from sort_cases import check_group_sort_equals_alone, check_sort_keeps_values


def test_sort_keeps_every_particle_oracle():
    check_sort_keeps_values(OracleEngine, nsteps=4, interval=2)


def test_sort_in_asynchronous_steps_oracle():
    check_sort_keeps_values(OracleEngine, nsteps=3, interval=3, use_async=True)


def test_sort_arguments_oracle():
    e = OracleEngine(make_config(16, species=[{"n": 20}]))
    for interval, ratio in ((-1, 4), (1, 0), (1, 3)):
        with pytest.raises(LCSError) as ei:
            e.set_particle_sort(interval, ratio)
        assert ei.value.code == _abi.EINVAL
    e.set_particle_sort(0, 0)  # off: the ratio is not looked at
    e.close()
    f = OracleEngine(make_config(16, mode=_abi.MODE_FLOW))
    with pytest.raises(LCSError) as ei:
        f.set_particle_sort(1, 4)
    assert ei.value.code == _abi.EINVAL
    f.close()


def test_group_sorts_its_members_oracle():
    check_group_sort_equals_alone(OracleEngine, load_oracle())
