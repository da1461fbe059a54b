"""The multi-rank logic of bench.py on CPU: two gloo ranks run the same
collective steps as two GPU replicas (barrier, max and sum over ranks), the
whole-job value is all ranks' units over the slowest rank's time, and the
reference arm does its work on rank 0 only."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_WORKER = r"""
import json, os, sys
sys.path.insert(0, {root!r})
import torch
import torch.distributed as dist
import bench
rank = int(os.environ["RANK"]); world = int(os.environ["WORLD_SIZE"])
dist.init_process_group("gloo", init_method="env://", rank=rank, world_size=world)
barrier, mx, sm = bench.rank_ops(world, torch.device("cpu"))
barrier()
work = [3.0e9, 5.0e9][rank]       # units this rank processed
ms = [1500.0, 2000.0][rank]       # its device time
out = {{"rank": rank, "max": mx(float(rank + 1)), "sum": sm(float(rank + 1)),
        "value": bench.replica_value(work, ms, mx, sm)}}
barrier()
dist.destroy_process_group()
print(json.dumps(out))
"""


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run_ranks(code: str, world: int = 2, extra_env=None):
    port = _free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE=str(world), LOCAL_RANK=str(r), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        env.update(extra_env or {})
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            o, e = p.communicate(timeout=180)
        except subprocess.TimeoutExpired:
            p.kill()
            raise
        assert p.returncode == 0, e[-2000:]
        outs.append(o)
    return outs


def test_replica_collectives_on_two_gloo_ranks():
    outs = [json.loads(o.strip().splitlines()[-1]) for o in _run_ranks(_WORKER.format(root=ROOT))]
    for o in outs:
        assert o["max"] == 2.0 and o["sum"] == 3.0
        # (3e9 + 5e9) units over the slower rank's 2.0 s
        assert o["value"] == pytest.approx(4.0e9, rel=1e-12)


def test_rank_ops_are_identity_on_one_rank():
    sys.path.insert(0, ROOT)
    import bench
    import torch
    barrier, mx, sm = bench.rank_ops(1, torch.device("cpu"))
    barrier()
    assert mx(2.5) == 2.5 and sm(2.5) == 2.5
    assert bench.replica_value(1.0e9, 500.0, mx, sm) == pytest.approx(2.0e9)


def test_reference_arm_runs_on_rank_zero_only():
    # a non-zero rank of the reference arm exits 0 at once, printing nothing
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "3"], env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""


def test_sweep_shards_partition_the_instances():
    sys.path.insert(0, ROOT)
    import bench
    for world in (1, 2, 3, 8):
        parts = [bench.shard(256, world, r) for r in range(world)]
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(256))
        assert max(len(p) for p in parts) - min(len(p) for p in parts) <= 1


_GATHER_WORKER = r"""
import json, os, sys
sys.path.insert(0, {root!r})
import torch.distributed as dist
import bench
from enscdynamics_b200 import serving as S
rank = int(os.environ["RANK"]); world = int(os.environ["WORLD_SIZE"])
dist.init_process_group("gloo", init_method="env://", rank=rank, world_size=world)
# rank r served requests r, r + world, ...: arrival i / 10 s, latency 1 + i s
mine = [S.Outcome(i, i / 10.0, admitted=i / 10.0, finished=i / 10.0 + 1.0 + i, cycles=100, elements=1000)
        for i in range(rank, 10, world)]
allo = bench.gather_outcomes(mine, world)
summ = S.summarize(allo)
dist.destroy_process_group()
print(json.dumps({{"indices": [o.index for o in allo], "requests": summ["requests"],
                   "p50": summ["p50_latency_s"], "makespan": summ["makespan_s"]}}))
"""


def test_serving_outcomes_are_gathered_over_ranks():
    """The multi-GPU serving leg shards the stream by request index; every
    rank ends with the whole stream's outcomes for its percentiles."""
    outs = [json.loads(o.strip().splitlines()[-1]) for o in _run_ranks(_GATHER_WORKER.format(root=ROOT))]
    for o in outs:
        assert o["indices"] == list(range(10)) and o["requests"] == 10
        assert o["p50"] == pytest.approx(5.5)          # latencies 1..10 s
        assert o["makespan"] == pytest.approx(10.9)    # first arrival 0, last finish 0.9 + 10
