"""Multi-rank host logic of the benchmark on CPU (gloo, world size 2).

On several GPUs every rank solves its own system (weak scaling, no data-path
collective), and the batched workload is sharded over the ranks by a
cost-balanced partition of its independent systems; ranks meet only at
barriers, at the max-over-ranks reduction of the timing and at the gather of
the batch energies.  These tests run that logic with the gloo backend."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r'''
import os, sys, json
sys.path.insert(0, {root!r})
import bench
rank, world, local = bench.dist_init(2)
# each rank reports a different time; everybody must see the max
t = 0.5 + rank
m = bench.dist_max(t, world)
bench.barrier(world)
# systems are seeded per rank: distinct models, identical shapes
from xatu_b200.synthetic import synthetic_hexagonal
h = synthetic_hexagonal(seed=1234 + rank).systemInfo.hamiltonian
print(json.dumps({{"rank": rank, "world": world, "max": m, "h00": float(abs(h[0, 0, 0])), "shape": list(h.shape)}}))
import torch.distributed as dist
dist.destroy_process_group()
'''


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_rank_max_and_barrier(tmp_path):
    script = tmp_path / "worker.py"
    script.write_text(WORKER.format(root=ROOT))
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE="2", LOCAL_RANK=str(r), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err
        outs.append(__import__("json").loads(out.strip().splitlines()[-1]))
    assert all(o["world"] == 2 for o in outs)
    assert all(o["max"] == pytest.approx(1.5) for o in outs)
    assert outs[0]["shape"] == outs[1]["shape"]
    assert outs[0]["h00"] != outs[1]["h00"]


def test_reference_arm_rank_gating(monkeypatch):
    """Under torchrun only rank 0 of the reference arm does work; other ranks return at once."""
    import types
    import bench
    calls = []

    class Fake:
        def __init__(self, ncell):
            calls.append(ncell)

    monkeypatch.setattr(bench, "dist_init", lambda n: (1, 2, 1))
    monkeypatch.setattr(bench, "CpuReference", Fake)
    bench.run_reference(types.SimpleNamespace(gpus=2, warmup=0, steps=1, ncell=6))
    assert calls == []


SHARD_WORKER = r'''
import os, sys, json
sys.path.insert(0, {root!r})
import bench
import torch.distributed as dist
rank, world, local = bench.dist_init(2)
specs, costs, mine = bench.batch_shard(64, rank, world)
parts = [None] * world
dist.all_gather_object(parts, {{"members": mine, "cost": int(sum(costs[i] for i in mine))}})
print(json.dumps({{"rank": rank, "parts": parts, "total": int(sum(costs))}}))
dist.destroy_process_group()
'''


def test_two_rank_batch_shards(tmp_path):
    """Every member of the 64-system batch lands on exactly one rank, both ranks compute the same
    partition, and the sum of N^2 per rank is balanced."""
    script = tmp_path / "shard_worker.py"
    script.write_text(SHARD_WORKER.format(root=ROOT))
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE="2", LOCAL_RANK=str(r), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err
        outs.append(__import__("json").loads(out.strip().splitlines()[-1]))
    assert outs[0]["parts"] == outs[1]["parts"]
    parts = outs[0]["parts"]
    members = sorted(i for p in parts for i in p["members"])
    assert members == list(range(64))
    loads = [p["cost"] for p in parts]
    assert sum(loads) == outs[0]["total"]
    assert max(loads) / (sum(loads) / 2) < 1.05


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_shard_members_partition(world):
    """The greedy partition covers every member once, is deterministic, and keeps the heaviest rank within
    the largest single member of the average (the classic bound of the greedy rule)."""
    from xatu_b200.batch import member_cost, shard_members
    from xatu_b200.synthetic import batch_workload
    specs = batch_workload(count=64)
    costs = [member_cost(s["ncell"] ** 2, s["nv"], s["nc"]) for s in specs]
    parts = shard_members(costs, world)
    assert parts == shard_members(costs, world)
    assert sorted(i for p in parts for i in p) == list(range(64))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) <= sum(costs) / world + max(costs)
