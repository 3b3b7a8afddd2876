"""The batching and serving forms over the CPU oracle (no GPU): the scheduler,
admission by footprint, slot limits, async steps and result hand-back are host
logic, identical over either library.  tests/test_gpu_serve.py runs the same
cases over the CUDA library."""

from oracle_engine import OracleEngine, load_oracle
from serve_cases import (check_async_equals_step, check_batch_equals_members_alone, check_group_equals_members_alone,
                         check_server, group_configs)


def test_async_steps_equal_step_oracle():
    check_async_equals_step(OracleEngine, load_oracle())


def test_batch_members_equal_solo_runs_oracle():
    check_batch_equals_members_alone(OracleEngine, load_oracle(), nsteps=2)


def test_server_continuous_batching_oracle():
    check_server(OracleEngine, load_oracle())


def test_group_members_equal_solo_runs_oracle():
    check_group_equals_members_alone(OracleEngine, load_oracle(), count=3, nsteps=1, n=16)


def test_batch_of_one_shape_oracle():
    check_batch_equals_members_alone(OracleEngine, load_oracle(), nsteps=1, cfgs=group_configs(n=16, count=3))
