"""The multi-process (replicas) path of bench.py, on CPU with the gloo backend.

bench.py runs one independent replica of the time step per GPU: each rank
holds its own seeded 256^3 state, there is no exchange on the data path, and
the only collectives are the barriers around the timed region and the
max-over-ranks of the device time.  These tests run that plumbing with two
ranks on the host (127.0.0.1 rendezvous) and check the reference arm's rank
rule (rank 0 alone measures and prints; other ranks exit 0 without work).
"""

import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_SCRIPT = r"""
import json, os, sys
sys.path.insert(0, {root!r})
import bench
world, rank, local = bench.dist_setup()
assert world == 2 and rank == int(os.environ["RANK"])
bench.barrier(world)
# device time of this rank's replica: rank 1 is the slow one
ms = 10.0 + 5.0 * rank
ms_max = bench.reduce_max(ms, world)
n3, steps = 256.0 ** 3, 4
value = world * n3 * steps / (ms_max / 1e3) / 1e6  # bench.py's whole-job aggregate
bench.barrier(world)
import torch.distributed as dist
dist.destroy_process_group()
print(json.dumps({{"rank": rank, "ms_max": ms_max, "value": value}}), flush=True)
"""


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def run_ranks(script, world=2, extra_env=None, timeout=120):
    port = free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        env.update(extra_env or {})
        procs.append(subprocess.Popen([sys.executable, "-c", script], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            o, e = p.communicate(timeout=timeout)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
        assert p.returncode == 0, e[-2000:]
        outs.append(o)
    return outs


def test_two_gloo_ranks_take_the_max_device_time():
    outs = run_ranks(RANK_SCRIPT.format(root=ROOT))
    lines = [json.loads(o.strip().splitlines()[-1]) for o in outs]
    assert sorted(ln["rank"] for ln in lines) == [0, 1]
    for ln in lines:
        assert ln["ms_max"] == 15.0  # every rank sees the slowest replica's time
        assert ln["value"] == pytest.approx(2 * 256.0 ** 3 * 4 / 0.015 / 1e6)


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2", MASTER_ADDR="127.0.0.1", MASTER_PORT="1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""


def test_reference_arm_rank0_prints_one_line():
    env = dict(os.environ, RANK="0", LOCAL_RANK="0", WORLD_SIZE="2", LCS_REFERENCE_BUDGET_S="0.1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--workload", "lp128"], env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0
